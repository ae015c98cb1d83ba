"""GPU shading parity against the oracle (itself pinned to the reference's
main_gpu.cu kernels run on the host). The kernels and the oracle share this
library's FP32 sincos for the AO/PT sample directions, so occlusion counts
and path-traced accumulators must agree exactly; the packed pixels go
through powf, whose last-ulp differences may move a channel by at most 1."""
import os

import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def channels(p):
    return np.stack([(p >> s) & 255 for s in (0, 8, 16, 24)], -1).astype(np.int32)


def gpu_ao(b, t, cam, w, h, ns, radius, seed=12345, sobol=1, traversal=mb.TRAVERSAL_STACKFREE, leaf_tris=None):
    import torch
    px = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    occ = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    stats = torch.zeros(8, dtype=torch.int64, device="cuda")
    mb.render_ao(px, (w, h), mb.RayGenerator.from_array(cam), b.m_rootNode, b.m_internals, t, sobol, ns, radius,
                 seed, occluded=occ, stats=stats, traversal=traversal, leaf_triangles=leaf_tris)
    torch.cuda.synchronize()
    st = G.host(stats)
    return G.host(px, np.uint32), G.host(occ, np.uint32), (int(st[0]), int(st[1]), int(st[2]))


def check_ao(gpu_px, gpu_occ, ref_px, ref_occ):
    np.testing.assert_array_equal(gpu_occ, ref_occ)
    d = np.abs(channels(gpu_px) - channels(ref_px))
    assert d.max() <= 1
    assert (d > 0).mean() < 1e-3


@pytest.mark.parametrize("sobol", [1, 0])
def test_ao_small_scene(cuda, sobol):
    g = np.load(os.path.join(GOLD, "builds.npz"))
    tris = g["small_scene/tris"]
    b, t, out = G.build(tris)
    s = np.load(os.path.join(GOLD, "shading.npz"))
    w, h = s["size"].tolist()
    cam = s["camera"]
    px, occ, st = gpu_ao(b, t, cam, w, h, 16, 1.0, 12345, sobol)
    rpx, rocc = O.render_ao(cam, out["root"], out["nodes"], tris, w, h, 16, 1.0, 12345, sobol, trig=1)
    check_ao(px, occ, rpx, rocc)
    assert st[0] == w * h + 16 * int((occ != 0xFFFFFFFF).sum())


def test_ao_heightfield_config(cuda):
    """212,992-triangle heightfield + icospheres, 512 x 512, 16 Owen-Sobol AO
    rays per hit, radius 0.25."""
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = O.lookat(eye, c, up, fovy, 512, 512)
    px, occ, st = gpu_ao(b, t, cam, 512, 512, 16, 0.25)
    rpx, rocc, cnt = O.render_ao(cam, out["root"], out["nodes"], tris, 512, 512, 16, 0.25, 12345, 1, trig=1,
                                 counters=True)
    check_ao(px, occ, rpx, rocc)
    # rays, internal-node visits and triangle tests: the traffic model of the roofline
    assert st == (int(cnt[2]), int(cnt[0]), int(cnt[1]))


@pytest.mark.parametrize("sobol", [1, 0])
def test_ao_replay_walk_equals_stackfree(cuda, sobol):
    """The replay form (replay walk, AO rays starting at the deepest node that
    holds every leaf within the AO radius) gives every pixel's occlusion count
    of the stack-free walk (which the oracle pins), with fewer node visits."""
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = O.lookat(eye, c, up, fovy, 512, 512)
    px0, occ0, st0 = gpu_ao(b, t, cam, 512, 512, 16, 0.25, sobol=sobol)
    px1, occ1, st1 = gpu_ao(b, t, cam, 512, 512, 16, 0.25, sobol=sobol, traversal=mb.TRAVERSAL_REPLAY)
    np.testing.assert_array_equal(occ1, occ0)
    np.testing.assert_array_equal(px1, px0)
    # the same rays; AO rays start below the root (at the node whose subtree holds every
    # leaf within their reach), so they test a subset of the same leaves, in the same order
    assert st1[0] == st0[0] and st1[2] <= st0[2]
    assert st1[1] < st0[1]
    # the same walk over leaf-ordered 48-byte triangles
    lt = mb.leaf_triangles(b, t)
    px2, occ2, st2 = gpu_ao(b, t, cam, 512, 512, 16, 0.25, sobol=sobol, traversal=mb.TRAVERSAL_REPLAY, leaf_tris=lt)
    np.testing.assert_array_equal(occ2, occ0)
    np.testing.assert_array_equal(px2, px0)
    assert st2 == st1


def test_ao_soup_config_full_frame(cuda):
    """The bench's workload: 4M-triangle soup, 1920 x 1080, 64 AO rays per hit,
    radius 0.1. The oracle renders the whole frame (all host threads); every
    pixel's occlusion count and packed colour of the plain form (the
    reference's stack-free walk), the replay walk, the 4-wide tree (the
    bench's chosen form) and its 8-bit quantised slots must be the oracle's."""
    import torch
    tris = scenes.gaussian_soup()
    b, t, out = G.build(tris)
    eye, c, up, fovy = scenes.camera_soup()
    w, h = 1920, 1080
    cam = O.lookat(eye, c, up, fovy, w, h)
    rpx, rocc = O.render_ao(cam, out["root"], out["nodes"], tris, w, h, 64, 0.1, 12345, 1, trig=1)
    assert (rocc != 0xFFFFFFFF).mean() > 0.05
    px, occ, _ = gpu_ao(b, t, cam, w, h, 64, 0.1)
    check_ao(px, occ, rpx, rocc)
    px, occ, _ = gpu_ao(b, t, cam, w, h, 64, 0.1, traversal=mb.TRAVERSAL_REPLAY, leaf_tris=mb.leaf_triangles(b, t))
    check_ao(px, occ, rpx, rocc)
    wide = mb.WideBVH.from_builder(b, t).quantise()
    for quantised in (False, True):
        dpx = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        docc = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        mb.render_ao_wide(dpx, (w, h), mb.RayGenerator.from_array(cam), wide, 1, 64, 0.1, 12345, occluded=docc,
                          quantised=quantised)
        torch.cuda.synchronize()
        assert int(G.host(wide.status)[0]) == 0
        check_ao(G.host(dpx, np.uint32), G.host(docc, np.uint32), rpx, rocc)


def test_normal_matches_golden_and_oracle(cuda):
    import torch
    g = np.load(os.path.join(GOLD, "builds.npz"))
    tris = g["small_scene/tris"]
    b, t, out = G.build(tris)
    s = np.load(os.path.join(GOLD, "shading.npz"))
    w, h = s["size"].tolist()
    px = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    mb.render_normal(px, (w, h), mb.RayGenerator.from_array(s["camera"]), b.m_rootNode, b.m_internals, t)
    got = G.host(px, np.uint32)
    d = np.abs(channels(got) - channels(s["normal"]))
    assert d.max() == 0


@pytest.mark.parametrize("sobol", [1, 0])
def test_pt_small_scene(cuda, sobol):
    import torch
    g = np.load(os.path.join(GOLD, "builds.npz"))
    tris = g["small_scene/tris"]
    b, t, out = G.build(tris)
    s = np.load(os.path.join(GOLD, "shading.npz"))
    w, h = s["size"].tolist()
    cam = s["camera"]
    attribs = s["attribs"]
    acc = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda")
    at = G.dev(attribs)
    ref = np.zeros((w * h, 4), np.float32)
    for _ in range(3):
        mb.render_pt(acc, (w, h), mb.RayGenerator.from_array(cam), b.m_rootNode, b.m_internals, t, at, sobol)
        O.render_pt(ref, cam, out["root"], out["nodes"], tris, attribs, w, h, sobol, trig=1)
    got = G.host(acc)
    np.testing.assert_array_equal(got, ref)
    px = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    mb.pack(px, acc, w * h)
    d = np.abs(channels(G.host(px, np.uint32)) - channels(O.pack(ref, w * h)))
    assert d.max() <= 1


def test_pt_heightfield(cuda):
    import torch
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    attribs = scenes.pt_attributes(len(tris), light_fraction=0.01)
    eye, c, up, fovy = scenes.camera_heightfield()
    w, h = 96, 96
    cam = O.lookat(eye, c, up, fovy, w, h)
    acc = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda")
    at = G.dev(attribs)
    ref = np.zeros((w * h, 4), np.float32)
    for _ in range(2):
        mb.render_pt(acc, (w, h), mb.RayGenerator.from_array(cam), b.m_rootNode, b.m_internals, t, at, 1)
        O.render_pt(ref, cam, out["root"], out["nodes"], tris, attribs, w, h, 1, trig=1)
    np.testing.assert_array_equal(G.host(acc), ref)
    assert ref[:, 0].sum() > 0


def test_pt_replay_walk_equals_stackfree(cuda):
    """mlbvh_render_pt_ex with the replay walk (with and without the
    leaf-ordered triangle copy) gives the stack-free walk's accumulators bit
    for bit over several progressive passes: the same Hit records per ray."""
    import torch
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    attribs = scenes.pt_attributes(len(tris), light_fraction=0.01)
    eye, c, up, fovy = scenes.camera_heightfield()
    w, h = 128, 96
    cam = mb.RayGenerator.from_array(O.lookat(eye, c, up, fovy, w, h))
    at = G.dev(attribs)
    lt = mb.leaf_triangles(b, t)
    accs = [torch.zeros((w * h, 4), dtype=torch.float32, device="cuda") for _ in range(3)]
    for sobol in (1, 0):
        for a in accs:
            a.zero_()
        for _ in range(3):
            mb.render_pt(accs[0], (w, h), cam, b.m_rootNode, b.m_internals, t, at, sobol)
            mb.render_pt(accs[1], (w, h), cam, b.m_rootNode, b.m_internals, t, at, sobol,
                         traversal=mb.TRAVERSAL_REPLAY)
            mb.render_pt(accs[2], (w, h), cam, b.m_rootNode, b.m_internals, t, at, sobol,
                         traversal=mb.TRAVERSAL_REPLAY, leaf_triangles=lt)
        torch.cuda.synchronize()
        assert torch.equal(accs[1], accs[0]) and torch.equal(accs[2], accs[0])
        assert float(accs[0][:, 0].sum()) > 0


def test_pt_obj_scene(cuda, tmp_path):
    """A scene read from OBJ / MTL (mlbvh_obj_load): the Cornell-style test
    box with a lamp, path traced on the GPU, equals the oracle's pt
    accumulators bit for bit over several passes."""
    import torch
    import _objscene
    tris, attribs = mb.load_obj(_objscene.write_cornell(str(tmp_path)))
    b, t, out = G.build(tris)
    w, h = 96, 72
    cam = O.lookat((0, 1, 3.5), (0, 1, 0), (0, 1, 0), np.float32(np.deg2rad(45.0)), w, h)
    acc = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda")
    at = G.dev(attribs)
    ref = np.zeros((w * h, 4), np.float32)
    for _ in range(4):
        mb.render_pt(acc, (w, h), mb.RayGenerator.from_array(cam), b.m_rootNode, b.m_internals, t, at, 1)
        O.render_pt(ref, cam, out["root"], out["nodes"], tris, attribs, w, h, 1, trig=1)
    np.testing.assert_array_equal(G.host(acc), ref)
    assert (ref[:, :3].sum(1) > 0).mean() > 0.02  # paths reach the lamp
