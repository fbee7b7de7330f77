"""Test-harness wrapper of the path-replay adjoint as a torch.autograd.Function.

The library itself exposes only the C-ABI (rumi_forward / rumi_backward /
rumi_scene_set_albedo / rumi_scene_set_volume); this module glues it to torch autograd
for the optimisation tests and the inverse-rendering benchmark.
"""
import torch


class PathTracedFilm(torch.autograd.Function):
    """film = render(albedo, medium) for one GpuScene and seed.

    albedo: (n_triangles, 3) float32 CUDA tensor (r, g, b), every triangle of the scene.
    medium: (7,) float32 CUDA tensor: sigma_s r,g,b, sigma_a r,g,b, g.
    Returns the film (H, W, 3) in B,G,R order holding per-pixel sample sums.

    grad_seed: the seed of the adjoint pass.  A loss that is nonlinear in the film (L2)
    needs it different from `seed`: the residual then comes from one set of paths and
    dfilm/dparams from an independent one, which makes the gradient unbiased (with the
    same paths the product picks up their covariance).  grad_seed == seed gives the exact
    derivative of this frame's <grad_film, film> (what finite differences under common
    random numbers measure)."""

    @staticmethod
    def forward(ctx, albedo, medium, gscene, spp, seed, grad_seed, grad_spp):
        albedo = albedo.detach().contiguous()
        m = medium.detach().cpu().tolist()
        torch.cuda.current_stream().synchronize()
        gscene.set_albedo(device_ptr=albedo.data_ptr())
        gscene.set_volume(m[0:3], m[3:6], m[6])
        film = torch.empty((gscene.height, gscene.width, 3), dtype=torch.float32, device=albedo.device)
        gscene.forward(spp=spp, seed=seed, film_device_ptr=film.data_ptr())
        ctx.gscene, ctx.spp, ctx.seed = gscene, grad_spp or spp, grad_seed
        ctx.scale = float(spp) / float(ctx.spp)
        ctx.shape_a = albedo.shape
        return film

    @staticmethod
    def backward(ctx, grad_film):
        g = grad_film.detach().contiguous()
        ga = torch.empty(ctx.shape_a, dtype=torch.float32, device=g.device)
        gv = torch.empty(7, dtype=torch.float32, device=g.device)
        torch.cuda.current_stream().synchronize()
        ctx.gscene.backward_device(g.data_ptr(), ga.data_ptr(), gv.data_ptr(), spp=ctx.spp, seed=ctx.seed)
        if ctx.scale != 1.0:  # the film holds sums of spp samples; the adjoint traced grad_spp
            ga *= ctx.scale
            gv *= ctx.scale
        return ga, gv, None, None, None, None, None


def render(albedo, medium, gscene, spp, seed, grad_seed=None, grad_spp=None):
    """Differentiable render; grad_seed defaults to a seed decorrelated from `seed`;
    grad_spp (default spp) is the number of samples per pixel the adjoint pass traces."""
    return PathTracedFilm.apply(albedo, medium, gscene, spp, seed,
                                seed + 0x5BD1E995 if grad_seed is None else grad_seed, grad_spp)


def _camera_hits(gscene, scene, sub):
    """Closest-hit primitive of sub x sub rays per pixel through the pinhole
    (Pinhole::CastViewRay's pixel grid, src/Camera/pinhole.cpp:97-136): (H*sub, W*sub)."""
    import numpy as np
    cam, img = scene.camera, scene.image
    W, H = img.width, img.height
    tan = np.tan(np.radians(cam.fov) * 0.5)
    xs = (np.arange(W * sub) + 0.5) / sub
    ys = (np.arange(H * sub) + 0.5) / sub
    X, Y = np.meshgrid(xs, ys)
    dx = -(X - W / 2) / (W / 2) * tan
    dy = -(Y - H / 2) / (H / 2) * tan * cam.y_ratio
    d = np.stack([dx, dy, np.ones_like(dx)], -1).reshape(-1, 3)
    m = np.asarray(cam.basis, np.float64).reshape(4, 4)[:3, :3]
    d = d @ m.T
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((d.shape[0], 7), np.float32)
    rays[:, 0:3] = np.asarray(cam.position, np.float32)
    rays[:, 3:6] = d
    rays[:, 6] = 3.4e38
    _, prim, _, _ = gscene.trace(rays)
    return prim.reshape(H * sub, W * sub)


def footprint_albedo_rmse(gscene, scene, first_mesh, n_mesh, albedo, hidden, sub=4):
    """RMSE, over the pixels that see the mesh, of the albedo averaged over each pixel's
    footprint (the mean over its sub x sub camera rays of the albedo of the triangle each
    hits) -- the part of the per-triangle albedo an image of this resolution observes.
    albedo, hidden: (n_mesh, 3) tensors.  Returns a float."""
    import numpy as np
    import torch
    prim = _camera_hits(gscene, scene, sub) - first_mesh
    H, W = prim.shape[0] // sub, prim.shape[1] // sub
    on = (prim >= 0) & (prim < n_mesh)
    ids = torch.from_numpy(np.where(on, prim, 0).astype(np.int64)).to(albedo.device)
    mask = torch.from_numpy(on).to(albedo.device)
    diff = (albedo - hidden)[ids] * mask[..., None]
    cnt = mask.reshape(H, sub, W, sub).sum((1, 3))
    fp = diff.reshape(H, sub, W, sub, 3).sum((1, 3)) / cnt.clamp(min=1)[..., None]
    seen = cnt == sub * sub  # pixels wholly on the mesh
    return float((fp[seen] ** 2).mean().sqrt())


def visible_triangles(gscene, scene, first_mesh, n_mesh, sub=4, min_pixels=1.0):
    """Mesh triangles the camera sees: closest hits of sub x sub rays per pixel through the
    pinhole (Pinhole::CastViewRay's pixel grid, src/Camera/pinhole.cpp:97-136) counted per
    triangle; a triangle covering at least `min_pixels` pixels is visible.  first_mesh:
    canonical id of the mesh's first triangle.  Returns a boolean mask (n_mesh,)."""
    import numpy as np
    prim = _camera_hits(gscene, scene, sub).reshape(-1)
    k = prim - first_mesh
    k = k[(prim >= 0) & (k >= 0) & (k < n_mesh)]
    cover = np.bincount(k, minlength=n_mesh) / float(sub * sub)
    return cover >= min_pixels
