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
    def forward(ctx, albedo, medium, gscene, spp, seed, grad_seed):
        albedo = albedo.detach().contiguous()
        m = medium.detach().cpu().tolist()
        torch.cuda.current_stream().synchronize()
        gscene.set_albedo(device_ptr=albedo.data_ptr())
        gscene.set_volume(m[0:3], m[3:6], m[6])
        film = torch.empty((gscene.height, gscene.width, 3), dtype=torch.float32, device=albedo.device)
        gscene.forward(spp=spp, seed=seed, film_device_ptr=film.data_ptr())
        ctx.gscene, ctx.spp, ctx.seed = gscene, spp, grad_seed
        ctx.shape_a = albedo.shape
        return film

    @staticmethod
    def backward(ctx, grad_film):
        g = grad_film.detach().contiguous()
        ga = torch.empty(ctx.shape_a, dtype=torch.float32, device=g.device)
        gv = torch.empty(7, dtype=torch.float32, device=g.device)
        torch.cuda.current_stream().synchronize()
        ctx.gscene.backward_device(g.data_ptr(), ga.data_ptr(), gv.data_ptr(), spp=ctx.spp, seed=ctx.seed)
        return ga, gv, None, None, None, None


def render(albedo, medium, gscene, spp, seed, grad_seed=None):
    """Differentiable render; grad_seed defaults to a seed decorrelated from `seed`."""
    return PathTracedFilm.apply(albedo, medium, gscene, spp, seed,
                                seed + 0x5BD1E995 if grad_seed is None else grad_seed)
