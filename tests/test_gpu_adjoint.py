"""Differentiable path tracing and its path-replay adjoint (no reference
counterpart). The GPU image must equal the oracle's FP32 image bit for bit
(same paths, same float operations); the GPU gradient must match the FP64
host adjoint and central finite differences (eps 1e-3, FP64 host renders) to
1e-3 relative on 32 triangles. The gradient flows through a
torch.autograd.Function used only here."""
import numpy as np
import pytest

import _diff as D
import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
REL_TOL = 1e-3


@pytest.fixture(scope="module")
def scene(cuda):
    tris, alb, em = scenes.diff_scene()
    b, t, out = G.build(tris)
    return tris, alb, em, b, t, out


def camera(w, h):
    eye, c, up, fovy = scenes.camera_heightfield()
    return mb.RayGenerator().lookat(eye, c, up, fovy, w, h)


def pick(grad, k=32, seed=5):
    """k triangles with gradients at least 1% of the largest (so relative
    errors are meaningful), chosen at random."""
    big = np.nonzero(np.abs(grad) > 0.01 * np.abs(grad).max())[0]
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(big, size=min(k, len(big)), replace=False))


@pytest.mark.parametrize("w,h,spp", [(96, 64, 8), (48, 40, 37), (40, 32, 64)])
def test_diff_render_matches_oracle(scene, w, h, spp):
    """Bit for bit: a pixel's samples are spread over the 32 lanes of a warp
    (lane l: samples l, l + 32, ...) and added as a pairwise tree in lane order;
    fewer samples than lanes, a count that is not a multiple of 32, and two
    samples per lane."""
    import torch
    tris, alb, em, b, t, out = scene
    cam = camera(w, h)
    img = torch.empty(w * h, dtype=torch.float32, device="cuda")
    mb.pt_diff_render(img, (w, h), cam, b, t, G.dev(alb), G.dev(em), spp, 3)
    ref = O.diff_render(out, tris, cam.as_array(), w, h, spp, 3, alb, em)
    np.testing.assert_array_equal(G.host(img), ref)
    assert (ref > 0).mean() > 0.05


def test_adjoint_matches_fp64_and_finite_differences(scene):
    import torch
    tris, alb, em, b, t, out = scene
    w, h, spp = 64, 64, 8
    cam = camera(w, h)
    cam_a = cam.as_array()
    target = O.diff_render(out, tris, cam_a, w, h, spp, 3, scenes.albedo(len(tris), 2), em, fp64=True)
    image = O.diff_render(out, tris, cam_a, w, h, spp, 3, alb, em, fp64=True)
    grad_image = 2.0 * (image - target)  # L2 loss sum_p (I_p - T_p)^2
    host = O.diff_adjoint(out, tris, cam_a, w, h, spp, 3, alb, em, grad_image)
    # the GPU adjoint through torch.autograd
    a = G.dev(alb).requires_grad_(True)
    img = D.render(a, b, t, G.dev(em), cam, w, h, spp, 3)
    img.backward(torch.from_numpy(grad_image.astype(np.float32)).cuda())
    gpu = G.host(a.grad).astype(np.float64)
    sel = pick(host)
    assert len(sel) == 32
    np.testing.assert_allclose(gpu[sel], host[sel], rtol=REL_TOL)
    eps = 1e-3
    a64 = alb.astype(np.float64)
    for tri in sel:
        up, dn = a64.copy(), a64.copy()
        up[tri] += eps
        dn[tri] -= eps
        lu = ((O.diff_render(out, tris, cam_a, w, h, spp, 3, up, em, fp64=True) - target) ** 2).sum()
        ld = ((O.diff_render(out, tris, cam_a, w, h, spp, 3, dn, em, fp64=True) - target) ** 2).sum()
        fd = (lu - ld) / (2 * eps)
        assert abs(host[tri] - fd) <= 1e-6 * abs(fd), (tri, host[tri], fd)
        assert abs(gpu[tri] - fd) <= REL_TOL * abs(fd), (tri, gpu[tri], fd)


def test_adjoint_full_config(scene):
    """512 x 512 at 64 spp, 3 bounces: GPU adjoint against the FP64 host
    adjoint on 32 triangles (the host re-traces all 67M rays)."""
    import torch
    tris, alb, em, b, t, out = scene
    w, h, spp = 512, 512, 64
    cam = camera(w, h)
    target = torch.empty(w * h, dtype=torch.float32, device="cuda")
    mb.pt_diff_render(target, (w, h), cam, b, t, G.dev(scenes.albedo(len(tris), 2)), G.dev(em), spp, 3)
    a = G.dev(alb).requires_grad_(True)
    img = D.render(a, b, t, G.dev(em), cam, w, h, spp, 3)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    gpu = G.host(a.grad).astype(np.float64)
    grad_image = (2.0 * (img - target)).detach().cpu().numpy().astype(np.float64)
    host = O.diff_adjoint(out, tris, cam.as_array(), w, h, spp, 3, alb, em, grad_image)
    sel = pick(host, seed=9)
    np.testing.assert_allclose(gpu[sel], host[sel], rtol=REL_TOL)
