"""Path-replay adjoint (rumi_forward / rumi_backward) on the inverse-rendering scene.

Albedo gradients are checked against central finite differences (h = 1e-3) of the GPU
renderer under common random numbers -- albedo drives no sampling decision, so the FD is
exact up to rounding and the adjoint must agree within 2% -- and against the REFERENCE
renderer's own finite-difference gradient (tests/golden/adjoint_fd_ref32.npz, generated
by tests/golden/make_golden.py with srand-fixed re-renders), statistically.  Medium
gradients (sigma_s, sigma_a, g drive the free-flight, absorption, shadow-transmittance
and phase-sampling decisions) are score-function estimates of the derivative of the
expected image; they are compared with CRN finite differences averaged over seeds,
within the combined standard error."""
import numpy as np
import pytest

import rumi_b200
from rumi_b200 import scenes

pytestmark = pytest.mark.gpu

REF_MEDIUM = dict(sigma_s=(0.45, 0.35, 0.25), sigma_a=(0.04, 0.06, 0.09), g=0.0)


def small(medium=None, size=32, spp=16, depth=4):
    return rumi_b200.GpuScene(scenes.inverse_rendering(size, size, spp, depth, levels=3, medium=medium))


def weighted(delta, film):
    return float((delta.astype(np.float64) * film).sum())


def test_forward_is_render_and_backward_is_deterministic():
    g = small()
    try:
        a, _ = g.forward(seed=9)
        b, _ = g.render(seed=9)
        assert np.array_equal(a, b)
        delta = np.random.default_rng(1).standard_normal(a.shape).astype(np.float32)
        ga1, gv1, st = g.backward(delta, seed=9)
        ga2, gv2, _ = g.backward(delta, seed=9)
        assert st["paths"] == 32 * 32 * 16
        assert np.isfinite(ga1).all() and np.isfinite(gv1).all()
        # atomics reorder float sums: equal to rounding
        np.testing.assert_allclose(ga1, ga2, rtol=1e-4, atol=1e-4 * np.abs(ga1).max())
        np.testing.assert_allclose(gv1, gv2, rtol=1e-4, atol=1e-4 * np.abs(gv1).max())
        z, zv, _ = g.backward(np.zeros_like(delta), seed=9)
        assert not z.any() and not zv.any()
        # linear in d_film
        ga3, gv3, _ = g.backward(2.0 * delta, seed=9)
        np.testing.assert_allclose(ga3, 2.0 * ga1, rtol=1e-4, atol=1e-4 * np.abs(ga1).max())
    finally:
        g.close()


def test_backward_reuses_the_kept_forward_radiance():
    """forward(keep=True) keeps every path's radiance; the next backward with the same seed,
    spp and depth skips its first pass (half the rays) and gives the same gradients; a
    different seed or a parameter update in between makes it trace the pass again."""
    g = small(medium=REF_MEDIUM)
    try:
        a, fst = g.forward(seed=9, wave_paths=5000)
        delta = np.random.default_rng(2).standard_normal(a.shape).astype(np.float32)
        ga0, gv0, st0 = g.backward(delta, seed=9, wave_paths=5000)
        k, _ = g.forward(seed=9, keep=True, wave_paths=3000)
        assert np.array_equal(a, k)
        ga1, gv1, st1 = g.backward(delta, seed=9, wave_paths=5000)
        assert st0["rays_extend"] == 2 * fst["rays_extend"]
        assert st1["rays_extend"] == fst["rays_extend"]  # the replay pass only
        np.testing.assert_allclose(ga1, ga0, rtol=1e-4, atol=1e-4 * np.abs(ga0).max())
        np.testing.assert_allclose(gv1, gv0, rtol=1e-4, atol=1e-4 * np.abs(gv0).max())
        _, _, st2 = g.backward(delta, seed=10)  # another frame: both passes
        assert st2["rays_extend"] > fst["rays_extend"]
        g.forward(seed=9, keep=True)
        g.set_albedo(np.full((g.flat.tri_vertices.shape[0], 3), 0.4, np.float32))
        _, _, st3 = g.backward(delta, seed=9)  # the scene changed: both passes
        assert st3["rays_extend"] > fst["rays_extend"]
    finally:
        g.close()


def test_albedo_gradient_matches_central_fd_under_crn():
    g = small()
    try:
        alb0 = g.flat.tri_albedo.copy()
        delta = np.random.default_rng(3).standard_normal((32, 32, 3)).astype(np.float32)
        ga, _, _ = g.backward(delta, seed=77, volume=False)
        h = 1e-3

        def fd_along(v):
            g.set_albedo(alb0 + h * v)
            fp = weighted(delta, g.forward(seed=77)[0])
            g.set_albedo(alb0 - h * v)
            fm = weighted(delta, g.forward(seed=77)[0])
            g.set_albedo(alb0)
            return (fp - fm) / (2 * h)

        big = np.abs(ga).max()
        top = np.argsort(-np.abs(ga).max(1))[:6]
        for t in top:
            for c in range(3):
                if abs(ga[t, c]) < 0.05 * big:
                    continue
                v = np.zeros_like(alb0)
                v[t, c] = 1.0
                fd = fd_along(v)
                assert abs(ga[t, c] - fd) <= 0.02 * abs(fd), (t, c, ga[t, c], fd)
        # a random direction over every triangle and channel
        v = np.random.default_rng(4).uniform(-1, 1, alb0.shape).astype(np.float32)
        fd = fd_along(v)
        adj = float((ga.astype(np.float64) * v).sum())
        assert abs(adj - fd) <= 0.02 * abs(fd), (adj, fd)
    finally:
        g.close()


def test_albedo_gradient_matches_reference_fd(golden):
    """Our adjoint of <delta, film> along 'the whole mesh's albedo in channel c', averaged
    over seeds, against the reference renderer's CRN finite differences of the same
    quantity (different random streams: compared within 4 combined standard errors)."""
    gf = golden("adjoint_fd_ref32.npz")
    delta = gf["delta"]
    g = small(medium=REF_MEDIUM)
    try:
        n_mesh = 4 * 4 ** 3
        rows = []
        for s in range(512):
            ga, _, _ = g.backward(delta, seed=5000 + s, volume=False)
            rows.append(ga[-n_mesh:].astype(np.float64).sum(0))
        rows = np.array(rows)
        mean, se = rows.mean(0), rows.std(0, ddof=1) / np.sqrt(rows.shape[0])
        for c in range(3):
            sig = np.sqrt(se[c] ** 2 + gf["stderr"][c] ** 2)
            assert abs(mean[c] - gf["mean"][c]) < 4.0 * sig, (c, mean, gf["mean"], se, gf["stderr"])
            assert sig < 0.05 * abs(gf["mean"][c])  # the comparison resolves 5% or better
    finally:
        g.close()


def test_medium_gradient_matches_fd_statistically():
    med = scenes.INVERSE_TARGET_MEDIUM
    g = small(medium=med, size=64, spp=64, depth=6)
    try:
        base = np.array(list(med["sigma_s"]) + list(med["sigma_a"]) + [med["g"]], np.float64)
        steps = np.maximum(0.1 * np.abs(base), 0.02)
        delta = (0.5 + np.random.default_rng(8).random((64, 64, 3))).astype(np.float32)
        adj, fd = [], []
        for s in range(48):
            seed = 300 + s
            _, gv, _ = g.backward(delta, seed=seed, albedo=False)
            adj.append(gv.astype(np.float64))
            row = []
            for k in range(7):
                vals = []
                for sgn in (1.0, -1.0):
                    v = base.copy()
                    v[k] += sgn * steps[k]
                    g.set_volume(v[0:3], v[3:6], v[6])
                    vals.append(weighted(delta, g.forward(seed=seed)[0]))
                row.append((vals[0] - vals[1]) / (2 * steps[k]))
            g.set_volume(base[0:3], base[3:6], base[6])
            fd.append(row)
        adj, fd = np.array(adj), np.array(fd)
        ma, mf = adj.mean(0), fd.mean(0)
        sa = adj.std(0, ddof=1) / np.sqrt(len(adj))
        sf = fd.std(0, ddof=1) / np.sqrt(len(fd))
        for k in range(7):
            # 4 combined standard errors plus 3% for the O(h^2) error of the wide FD step
            tol = 4.0 * np.sqrt(sa[k] ** 2 + sf[k] ** 2) + 0.03 * abs(mf[k])
            assert abs(ma[k] - mf[k]) < tol, (k, ma, mf, sa, sf)
    finally:
        g.close()


def test_backward_rejects_what_it_cannot_differentiate():
    g = rumi_b200.GpuScene(scenes.cornell_pt(16, 16, 4, 4))  # no per-triangle albedo, no medium
    try:
        d = np.ones((16, 16, 3), np.float32)
        with pytest.raises(rumi_b200._capi.RumiError):
            g.backward(d, seed=1, albedo=True, volume=False)
        with pytest.raises(rumi_b200._capi.RumiError):
            g.backward(d, seed=1, albedo=False, volume=True)
        with pytest.raises(rumi_b200._capi.RumiError):
            g.set_albedo(np.zeros((g.flat.tri_vertices.shape[0], 3), np.float32))
    finally:
        g.close()
    g = small()
    try:
        with pytest.raises(rumi_b200._capi.RumiError):
            g.set_volume((0.1, 0.1, 0.1), (0.0, 0.0, 0.0), 1.5)
    finally:
        g.close()


def test_inverse_rendering_reduces_loss_and_recovers_medium():
    """A short optimisation through the torch.autograd.Function wrapper: Adam on the mesh
    albedo and the medium from a wrong start.  The image loss, measured with a fixed-seed
    256-spp render against a 256-spp target, must fall; the medium coefficients must move
    toward the hidden target; and the albedo must approach the hidden one where the image
    observes it -- over the triangles that cover at least a pixel, and averaged over each
    pixel's footprint (the 256 triangles here are a few pixels each)."""
    import torch
    from adjoint_torch import render, visible_triangles, footprint_albedo_rmse
    size, spp, depth, eval_spp = 48, 16, 6, 256
    gt = rumi_b200.GpuScene(scenes.inverse_rendering(size, size, eval_spp, depth, levels=3))
    target = torch.from_numpy(gt.forward(seed=1)[0] / eval_spp).cuda()
    gt.close()
    n_mesh = 4 * 4 ** 3
    start = scenes.inverse_rendering(size, size, spp, depth, levels=3,
                                     albedo=np.full((n_mesh, 3), 0.5, np.float32),
                                     medium=scenes.INVERSE_START_MEDIUM)
    g = rumi_b200.GpuScene(start)
    try:
        alb_all = torch.from_numpy(start.flatten().tri_albedo.copy()).cuda()
        walls = alb_all[:-n_mesh].clone()
        mesh = torch.nn.Parameter(alb_all[-n_mesh:].clone())
        m0 = scenes.INVERSE_START_MEDIUM
        med = torch.nn.Parameter(torch.tensor(list(m0["sigma_s"]) + list(m0["sigma_a"]) + [m0["g"]],
                                              dtype=torch.float32, device="cuda"))

        def eval_loss():
            with torch.no_grad():
                film = render(torch.cat([walls, mesh]), med, g, eval_spp, 7) / eval_spp
                return float(((film - target) ** 2).mean())

        before = eval_loss()
        hidden = torch.from_numpy(scenes.random_albedo(n_mesh, 23)).cuda()
        first = alb_all.shape[0] - n_mesh
        vis = torch.from_numpy(visible_triangles(g, start, first, n_mesh)).cuda()
        assert int(vis.sum()) > 50
        vis0 = float(((mesh.detach() - hidden)[vis] ** 2).mean().sqrt())
        fp0 = footprint_albedo_rmse(g, start, first, n_mesh, mesh.detach(), hidden)
        opt = torch.optim.Adam([mesh, med], lr=2e-2)
        for it in range(60):
            film = render(torch.cat([walls, mesh]), med, g, spp, 100 + it) / spp
            loss = ((film - target) ** 2).mean()
            opt.zero_grad()
            loss.backward()
            opt.step()
            with torch.no_grad():
                mesh.clamp_(0.01, 1.0)
                med[0:6].clamp_(1e-3, 5.0)
                med[6].clamp_(-0.9, 0.9)
        after = eval_loss()
        # Two independent 256-spp renders of the same scene differ by 0.00188 in this loss
        # (the oracle's figure for the target scene at seeds 1 and 7): 58% of `before` is
        # noise no parameter can remove.  16-spp gradients from a decorrelated seed are
        # noisy and the float atomics that sum them make each run's trajectory slightly
        # different; `after` fell to 0.6-0.85 of `before` over the runs observed.  The bound
        # 0.9 * before asks the removable part to shrink by a quarter.
        assert after < 0.9 * before, (before, after)
        vis1 = float(((mesh.detach() - hidden)[vis] ** 2).mean().sqrt())
        fp1 = footprint_albedo_rmse(g, start, first, n_mesh, mesh.detach(), hidden)
        assert vis1 < vis0 and fp1 < fp0, (vis0, vis1, fp0, fp1)
        t = scenes.INVERSE_TARGET_MEDIUM
        tgt = np.array(list(t["sigma_s"]) + list(t["sigma_a"]) + [t["g"]])
        m_start = np.array(list(m0["sigma_s"]) + list(m0["sigma_a"]) + [m0["g"]])
        m_end = med.detach().cpu().numpy()
        assert np.abs(m_end - tgt)[0:3].sum() < np.abs(m_start - tgt)[0:3].sum(), (m_end, tgt)
        assert abs(m_end[6] - tgt[6]) < abs(m_start[6] - tgt[6]), (m_end, tgt)
    finally:
        g.close()
