"""The quantised form (8-bit child boxes, 32-byte nodes; no reference
counterpart). The GPU conversion must equal the oracle's word for word, every
decoded box must contain its FP32 box, GPU traversal must equal the oracle's
quantised traversal bit for bit, and its hits must equal the FP32 tree's."""
import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu


def quantise_both(tris):
    b, t, out = G.build(tris)
    q = mb.QuantisedBVH.from_builder(b, t)
    n = len(tris)
    gq = dict(qnodes=G.host(q.qnodes, np.uint32)[: n - 1], parents=G.host(q.parents, np.uint32)[: n - 1],
              qtris=G.host(q.qtris, np.uint32), header=G.host(q.header, np.uint32))
    ref = O.quantise(out, tris)
    return b, t, out, q, gq, ref


@pytest.mark.parametrize("n", [1, 2, 3, 257, 4097, 100000])
def test_quantise_matches_oracle(cuda, n):
    tris = scenes.gaussian_soup(n, clusters=4, seed=300 + n)
    b, t, out, _, gq, ref = quantise_both(tris)
    for k in ("qnodes", "parents", "qtris", "header"):
        np.testing.assert_array_equal(gq[k], ref[k], err_msg=k)
    # mlbvh_leaf_triangles writes the same leaf-ordered triangles
    np.testing.assert_array_equal(G.host(mb.leaf_triangles(b, t), np.uint32), ref["qtris"])
    if n > 1:
        assert O.oracle().orc_check_quantised(O.P(out["nodes"]), n, O.P(gq["qnodes"]), O.P(gq["header"])) == 1


@pytest.fixture(scope="module")
def heightfield_q(cuda):
    tris = scenes.heightfield_icospheres()
    return (tris,) + quantise_both(tris)


def test_quantise_heightfield_conservative(heightfield_q):
    tris, _, _, out, _, gq, ref = heightfield_q
    for k in ("qnodes", "parents", "qtris", "header"):
        np.testing.assert_array_equal(gq[k], ref[k], err_msg=k)
    assert O.oracle().orc_check_quantised(O.P(out["nodes"]), len(tris), O.P(gq["qnodes"]), O.P(gq["header"])) == 1


@pytest.mark.parametrize("q", [0, 1])
def test_quantised_trace_heightfield(heightfield_q, q):
    tris, b, t, out, qb, gq, ref = heightfield_q
    rays = scenes.random_rays(200000, [-1, -0.3, -1], [1, 0.7, 1], seed=41)
    rays[1::3, 7] = 0.25
    got = G.host(mb.intersect_quantised(qb, G.dev(rays), q), np.uint32)
    np.testing.assert_array_equal(got, O.trace_quantised(ref, rays, q))
    plain = O.trace(out["nodes"], tris, out["root"], rays, q, 0)
    if q == 0:
        np.testing.assert_array_equal(got[:, 7], plain[:, 7])  # hit ids
        np.testing.assert_array_equal(got[:, 0], plain[:, 0])  # t
    else:
        np.testing.assert_array_equal(got[:, 7] == 0xFFFFFFFF, plain[:, 7] == 0xFFFFFFFF)


def test_quantised_ao_equals_plain(heightfield_q):
    import torch
    tris, b, t, out, qb, gq, ref = heightfield_q
    eye, c, up, fovy = scenes.camera_heightfield()
    w, h = 512, 512
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
    px0 = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    px1 = torch.zeros_like(px0)
    occ0 = torch.zeros_like(px0)
    occ1 = torch.zeros_like(px0)
    st = torch.zeros(8, dtype=torch.int64, device="cuda")
    mb.render_ao(px0, (w, h), cam, b.m_rootNode, b.m_internals, t, 1, 16, 0.25, occluded=occ0)
    mb.render_ao_quantised(px1, (w, h), cam, qb, 1, 16, 0.25, occluded=occ1, stats=st)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(G.host(occ1), G.host(occ0))
    np.testing.assert_array_equal(G.host(px1), G.host(px0))
    assert int(G.host(st)[0]) > w * h


def test_quantised_full_size_soup(cuda):
    tris = scenes.gaussian_soup()
    b, t, out, qb, gq, ref = quantise_both(tris)
    for k in ("qnodes", "parents", "qtris", "header"):
        np.testing.assert_array_equal(gq[k], ref[k], err_msg=k)
    rays = scenes.random_rays(100000, [0, 0, 0], [1, 1, 1], seed=19)
    rays[::2, 7] = 0.1
    got = G.host(mb.intersect_quantised(qb, G.dev(rays), 0), np.uint32)
    np.testing.assert_array_equal(got, O.trace_quantised(ref, rays, 0))
    plain = O.trace(out["nodes"], tris, out["root"], rays, 0, 0)
    np.testing.assert_array_equal(got[:, 7], plain[:, 7])


@pytest.mark.parametrize("q", [0, 1])
@pytest.mark.parametrize("depth", [0, 1, 4, 16])
def test_quantised_walks_match_oracle_with_counts(heightfield_q, q, depth):
    """Every walk (stack-free, or the replay walk with 1, 4 or 16 stack
    entries, overflowing to the stack-free walk) returns the oracle's Hit
    records, and per ray the oracle's node visits, triangle tests and parent
    loads for that walk."""
    import torch
    tris, b, t, out, qb, gq, ref = heightfield_q
    rays = scenes.random_rays(60000, [-1, -0.3, -1], [1, 0.7, 1], seed=43)
    rays[1::3, 7] = 0.25
    n = len(rays)
    counts = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
    got = G.host(mb.intersect_quantised(qb, G.dev(rays), q, stack_depth=depth, counts=counts), np.uint32)
    hits, nv, nt, nu = O.trace_quantised(ref, rays, q, counters=True, stack_depth=depth)
    np.testing.assert_array_equal(got, hits)
    c = G.host(counts, np.uint32)
    np.testing.assert_array_equal(c[:n], nv, err_msg="node visits")
    np.testing.assert_array_equal(c[n:2 * n], nt, err_msg="triangle tests")
    np.testing.assert_array_equal(c[2 * n:], nu, err_msg="parent loads")
    if depth == 0:
        np.testing.assert_array_equal(got, O.trace_quantised(ref, rays, q))


def test_quantised_replay_on_duplicate_chains(cuda):
    """A tree of long equal-key chains (deep) overflows small stacks: still the
    stack-free walk's Hit records."""
    tris = np.tile(scenes.gaussian_soup(3, seed=6), (3000, 1))
    b, t, out, qb, gq, ref = quantise_both(tris)
    rays = scenes.random_rays(20000, [0, 0, 0], [1, 1, 1], seed=44)
    want = O.trace_quantised(ref, rays, 0)
    for depth in (0, 1, 4, 16):
        got = G.host(mb.intersect_quantised(qb, G.dev(rays), 0, stack_depth=depth), np.uint32)
        np.testing.assert_array_equal(got, want, err_msg=f"depth {depth}")


def test_quantised_precision_config(cuda):
    """The precision configuration: the 4M-triangle soup, 1M camera rays of the
    1920x1080 frame, closest hits over the quantised and the FP32 tree: 100%
    hit-ID agreement, equal t, and every t within the FP64 bound."""
    from minimumlbvh_b200 import fp64check as F
    tris = scenes.gaussian_soup()
    b, t, out = G.build(tris)
    qb = mb.QuantisedBVH.from_builder(b, t)
    eye, c, up, fovy = scenes.camera_soup()
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, 1920, 1080)
    rays = scenes.camera_rays(cam.m_origin, cam.m_right, cam.m_up, 1920, 1080)
    plain = G.trace(b, t, rays, 0, 0)
    quant = G.host(mb.intersect_quantised(qb, G.dev(rays), 0), np.uint32)
    np.testing.assert_array_equal(quant[:, 7], plain[:, 7])
    np.testing.assert_array_equal(quant[:, 0], plain[:, 0])
    r = F.check_hits(tris, rays, quant)
    assert r["hits"] > 100000 and r["max_bound_ratio"] <= 1.0, r


@pytest.mark.parametrize("scale,status", [(1.0, 0), (1e20, 1), (1e37, 2)])
def test_quantised_status_paths_match_oracle(cuda, scale, status):
    """The three node tests of the quantised binary tree (the FMA form; the
    reference's slabs on the decoded boxes, for status bit 0 and for rays with
    a zero direction component; every box passing, for status bit 1) give the
    oracle's nodes, header, Hit records and per-ray counts on both walks, and
    the FP32 tree's closest hits."""
    import torch
    rng = np.random.default_rng(31)
    tris = ((rng.random((3000, 9)) - 0.5) * scale).astype(np.float32)
    b, t, out, qb, gq, ref = quantise_both(tris)
    for k in ("qnodes", "parents", "qtris", "header"):
        np.testing.assert_array_equal(gq[k], ref[k], err_msg=k)
    assert int(gq["header"][3]) == status
    rays = scenes.random_rays(3000, [-0.5 * scale] * 3, [0.5 * scale] * 3, seed=32)
    rays[0::3, 4 + (np.arange(0, 3000, 3) % 3)] = 0.0  # zero components: outside the FMA form's range
    n = len(rays)
    for depth in (0, 4):
        counts = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
        got = G.host(mb.intersect_quantised(qb, G.dev(rays), 0, stack_depth=depth, counts=counts), np.uint32)
        hits, nv, nt, nu = O.trace_quantised(ref, rays, 0, counters=True, stack_depth=depth)
        np.testing.assert_array_equal(got, hits)
        c = G.host(counts, np.uint32)
        np.testing.assert_array_equal(c[:n], nv, err_msg="node visits")
        np.testing.assert_array_equal(c[n:2 * n], nt, err_msg="triangle tests")
    plain = O.trace(out["nodes"], tris, out["root"], rays, 0, 0)
    np.testing.assert_array_equal(got[:, 7], plain[:, 7])
