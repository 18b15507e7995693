"""Differentiable physical-mode rendering for PyTorch.

render_physical(scene, cam, albedo, emission, ...) returns the physical-mode image as a tensor
that is differentiable with respect to the per-triangle albedo [num_triangles, 3] and the
per-object emission [num_objects, 3]. The backward pass is the library's path-replay adjoint
(swr_render_adjoint): it re-traces every camera path from its random-number counters instead of
keeping anything from the forward pass. With adjoint_seed = seed (the default) the gradient is the
exact derivative of the rendered Monte Carlo estimate; a different adjoint seed gives an
independent (decorrelated) gradient estimate.
"""
import torch

from . import _native as N


class _PhysicalRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, emission, scene, cam, width, height, spp, depth, seed, rr_depth, rr_survive,
                adjoint_seed):
        albedo = albedo.detach().contiguous()
        emission = emission.detach().contiguous()
        scene.set_albedo(albedo)
        scene.set_emission(emission)
        img = scene.render(cam, width, height, spp, depth, seed=seed, mode=N.MODE_PHYSICAL, rr_depth=rr_depth,
                           rr_survive=rr_survive)
        ctx.save_for_backward(albedo, emission)
        ctx.args = (scene, cam, width, height, spp, depth, seed if adjoint_seed is None else adjoint_seed,
                    rr_depth, rr_survive)
        return img

    @staticmethod
    def backward(ctx, grad):
        albedo, emission = ctx.saved_tensors
        scene, cam, width, height, spp, depth, seed, rr_depth, rr_survive = ctx.args
        # the scene is stateful: restore this forward's parameters before replaying its paths
        scene.set_albedo(albedo)
        scene.set_emission(emission)
        ga, ge = scene.render_adjoint(cam, width, height, spp, depth, grad.contiguous(), seed=seed,
                                      rr_depth=rr_depth, rr_survive=rr_survive)
        return ga, ge, None, None, None, None, None, None, None, None, None, None


def render_physical(scene, cam, albedo, emission, width, height, spp, depth, seed=0, rr_depth=0, rr_survive=1.0,
                    adjoint_seed=None):
    """Physical-mode image [height, width, 3], differentiable w.r.t. albedo and emission."""
    return _PhysicalRender.apply(albedo, emission, scene, cam, width, height, spp, depth, seed, rr_depth,
                                 rr_survive, adjoint_seed)
