"""torch.autograd wrapper of the differentiable path trace, for the tests
only: forward = mlbvh_pt_diff_render, backward = the path-replay adjoint
mlbvh_pt_diff_adjoint (paths re-traced from their seeds, nothing stored)."""
import torch

import minimumlbvh_b200 as mb


class PathTrace(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, builder, triangles, emission, camera, w, h, spp, bounces):
        image = torch.empty(w * h, dtype=torch.float32, device=albedo.device)
        mb.pt_diff_render(image, (w, h), camera, builder, triangles, albedo.contiguous(), emission, spp, bounces)
        ctx.save_for_backward(albedo)
        ctx.args = (builder, triangles, emission, camera, w, h, spp, bounces)
        return image

    @staticmethod
    def backward(ctx, grad_image):
        (albedo,) = ctx.saved_tensors
        builder, triangles, emission, camera, w, h, spp, bounces = ctx.args
        grad = torch.zeros_like(albedo)
        mb.pt_diff_adjoint(grad, grad_image.contiguous(), (w, h), camera, builder, triangles, albedo.contiguous(),
                           emission, spp, bounces)
        return grad, None, None, None, None, None, None, None, None


def render(albedo, builder, triangles, emission, camera, w, h, spp, bounces=3):
    return PathTrace.apply(albedo, builder, triangles, emission, camera, w, h, spp, bounces)
