"""Differentiable physical-mode rendering for PyTorch.

render_physical(scene, cam, albedo, emission, ...) returns the physical-mode image as a tensor
that is differentiable with respect to the per-triangle albedo [num_triangles, 3] and the
per-object emission [num_objects, 3]. The backward pass is the library's path-replay adjoint
(swr_render_adjoint): it re-traces every camera path from its random-number counters instead of
keeping anything from the forward pass. With adjoint_seed = seed (the default) the gradient is the
exact derivative of the rendered Monte Carlo estimate; a different adjoint seed gives an
independent (decorrelated) gradient estimate. render_physical_batch does the same for many scenes
at once through the batched primal (swr_render_batch) and adjoint (swr_render_adjoint_batch).
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


class _PhysicalRenderBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, jobs, adjoint_seeds, *params):
        params = [p.detach().contiguous() for p in params]
        for k, j in enumerate(jobs):
            j["scene"].set_albedo(params[2 * k])
            j["scene"].set_emission(params[2 * k + 1])
        imgs = batch.render([dict(j, mode=N.MODE_PHYSICAL) for j in jobs])
        ctx.save_for_backward(*params)
        ctx.batch, ctx.jobs, ctx.adjoint_seeds = batch, jobs, adjoint_seeds
        return tuple(imgs)

    @staticmethod
    def backward(ctx, *grads):
        params = ctx.saved_tensors
        adj = []
        for k, j in enumerate(ctx.jobs):
            j["scene"].set_albedo(params[2 * k])
            j["scene"].set_emission(params[2 * k + 1])
            g = grads[k]
            if g is None:
                g = torch.zeros((j["height"], j["width"], 3), dtype=torch.float32, device=params[2 * k].device)
            seed = j.get("seed", 0) if ctx.adjoint_seeds is None else ctx.adjoint_seeds[k]
            adj.append(dict(j, seed=seed, dl_dimage=g))
        out = ctx.batch.render_adjoint(adj)
        flat = []
        for ga, ge in out:
            flat += [ga, ge]
        return (None, None, None, *flat)


def render_physical_batch(batch, jobs, albedos, emissions, adjoint_seeds=None):
    """Physical-mode images of many scenes, one primal batch launch forward and one batched
    path-replay adjoint launch backward. jobs: dicts with scene, cam, width, height, spp, depth and
    optional seed, rr_depth, rr_survive; each job its own scene. albedos / emissions: per-job
    tensors [num_triangles, 3] / [num_objects, 3]. Returns a tuple of images [h, w, 3]."""
    if len({id(j["scene"]) for j in jobs}) != len(jobs):
        raise ValueError("render_physical_batch: each job needs its own scene")
    params = []
    for a, e in zip(albedos, emissions):
        params += [a, e]
    return _PhysicalRenderBatch.apply(batch, jobs, adjoint_seeds, *params)


class _PhysicalRenderSplit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, emission, scene, cam, width, height, spp, depth, seed, rr_depth, rr_survive, rank,
                world):
        from . import sharding
        albedo = albedo.detach().contiguous()
        emission = emission.detach().contiguous()
        scene.set_albedo(albedo)
        scene.set_emission(emission)
        part = sharding.scene_part_renderer(scene, cam, width, height, spp, depth, seed=seed, mode=N.MODE_PHYSICAL,
                                            rr_depth=rr_depth, rr_survive=rr_survive)
        img = sharding.render_split(part, width, height, spp, rank, world, split="spp", device=albedo.device)
        ctx.save_for_backward(albedo, emission)
        ctx.args = (scene, cam, width, height, spp, depth, seed, rr_depth, rr_survive, rank, world)
        return img

    @staticmethod
    def backward(ctx, grad):
        from . import sharding
        albedo, emission = ctx.saved_tensors
        scene, cam, width, height, spp, depth, seed, rr_depth, rr_survive, rank, world = ctx.args
        scene.set_albedo(albedo)
        scene.set_emission(emission)
        g = grad.contiguous()

        def part(s0, count):
            return scene.render_adjoint(cam, width, height, count, depth, g, seed=seed, rr_depth=rr_depth,
                                        rr_survive=rr_survive, sample_begin=s0, spp_total=spp)

        ga, ge = sharding.adjoint_split(part, spp, rank, world, [tuple(albedo.shape), tuple(emission.shape)],
                                        device=albedo.device)
        return ga, ge, None, None, None, None, None, None, None, None, None, None, None


def render_physical_split(scene, cam, albedo, emission, width, height, spp, depth, seed=0, rr_depth=0,
                          rr_survive=1.0, rank=0, world=1):
    """render_physical with one image's samples split over `world` ranks (one process per GPU,
    each holding the scene): the forward pass adds the ranks' sample ranges with one all_reduce
    of the image, the backward pass adds their path-replay gradients with one all_reduce per
    gradient, so every rank gets the whole image and the whole gradient (data-parallel inverse
    rendering with identical optimiser steps on every rank)."""
    return _PhysicalRenderSplit.apply(albedo, emission, scene, cam, width, height, spp, depth, seed, rr_depth,
                                      rr_survive, rank, world)
