"""torch.autograd wrapper of the closest-hit query (differentiation form).

    t, uv, normal, prim, geom, hit = trace(scene, origins, directions,
                                           vertices=v, centers=c, radii=r)

t, uv and normal are differentiable with respect to the ray origins and raw directions and to
the geometry tensors passed in (which must be the arrays the scene was committed from: the
forward pass runs on the committed scene).  The backward pass is bzr_adjoint_hit: it holds
each ray's hit primitive fixed and recomputes its intersection from the stored prim_id.
"""
from __future__ import annotations

import torch


class RayQuery(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scene, origins, directions, vertices, centers, radii):
        out = scene.intersectN(origins, directions)
        ctx.scene = scene
        ctx.fwd = {k: out[k] for k in ("t", "prim", "geom", "hit")}
        ctx.save_for_backward(origins, directions)
        ctx.n_vertices = 0 if vertices is None else vertices.shape[0]
        ctx.n_spheres = 0 if centers is None else centers.shape[0]
        ctx.mark_non_differentiable(out["prim"], out["geom"], out["hit"])
        return out["t"], out["uv"], out["normal"], out["prim"], out["geom"], out["hit"]

    @staticmethod
    def backward(ctx, g_t, g_uv, g_normal, *unused):
        origins, directions = ctx.saved_tensors
        g = ctx.scene.adjoint(origins, directions, ctx.fwd, grad_t=g_t, grad_uv=g_uv,
                              grad_normal=g_normal, n_vertices=ctx.n_vertices,
                              n_spheres=ctx.n_spheres)
        return (None, g["origins"], g["directions"], g["vertices"], g["centers"], g["radii"])


def trace(scene, origins, directions, vertices=None, centers=None, radii=None):
    return RayQuery.apply(scene, origins, directions, vertices, centers, radii)
