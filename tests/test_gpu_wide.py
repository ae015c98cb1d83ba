"""GPU parity of the 4-wide tree (mlbvh_build_wide, mlbvh_trace_wide,
mlbvh_render_ao_wide; no reference counterpart). Every slot must equal the
oracle's regrouping bit for bit; any-hit and closest-hit rays must return the
oracle's wide walk Hit records and counts exactly; any-hit rays hit exactly
when the stack-free walk (pinned to the reference's intersect_stackfree)
does, and closest-hit rays report its Hit records; AO over the wide
tree must give every pixel's occlusion count of mlbvh_render_ao."""
import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF


def _cases():
    yield "one", scenes.gaussian_soup(1, seed=1), ([0, 0, 0], [1, 1, 1])
    yield "two", scenes.gaussian_soup(2, seed=2), ([0, 0, 0], [1, 1, 1])
    yield "three", scenes.gaussian_soup(3, seed=3), ([0, 0, 0], [1, 1, 1])
    yield "soup", scenes.gaussian_soup(50000, clusters=8, seed=5), ([0, 0, 0], [1, 1, 1])
    yield "heightfield", scenes.heightfield_icospheres(), ([-1, -0.3, -1], [1, 0.7, 1])
    yield "duplicates", np.tile(scenes.gaussian_soup(3, seed=6), (400, 1)), ([0, 0, 0], [1, 1, 1])


@pytest.fixture(scope="module", params=[c[0] for c in _cases()])
def wcase(request, cuda):
    for name, tris, box in _cases():
        if name == request.param:
            b, t, out = G.build(tris)
            w = mb.WideBVH.from_builder(b, t)
            rays = scenes.random_rays(20000, box[0], box[1], seed=17)
            rays[1::3, 7] = 0.05
            return name, tris, b, t, out, w, rays


def test_wide_nodes_match_oracle(wcase):
    import torch
    _, tris, _, _, out, w, _ = wcase
    n = len(tris)
    torch.cuda.synchronize()
    if n == 1:
        return
    got = G.host(w.wide, np.uint32)[: n - 1]
    ref = O.build_wide(out["nodes"], n)
    bad = np.nonzero((got != ref).any(1))[0]
    assert bad.size == 0, f"{bad.size} slots differ, first {bad[:4]}"


def test_trace_wide_matches_oracle(wcase):
    import torch
    name, tris, b, t, out, w, rays = wcase
    r = G.dev(rays)
    counts = torch.zeros(3 * len(rays), dtype=torch.int32, device="cuda")
    hits = G.host(mb.intersect_wide(w, r, counts=counts), np.uint32)
    c = G.host(counts, np.uint32).reshape(3, -1)
    ref, nv, nt, nr = O.trace_wide(O.build_wide(out["nodes"], len(tris)), out["nodes"], tris, out["root"], rays)
    np.testing.assert_array_equal(hits, ref)
    np.testing.assert_array_equal(c[0], nv)
    np.testing.assert_array_equal(c[1], nt)
    np.testing.assert_array_equal(c[2], nr)
    plain = G.trace(b, t, rays, mb.RAY_QUERY_ANY)
    np.testing.assert_array_equal(hits[:, 7] == MISS, plain[:, 7] == MISS)


def test_trace_wide_restarts_on_stack_overflow(cuda):
    """Rays parallel to a triangle duplicated 400 times: the wide stack
    overflows and the ray restarts with the stack-free walk (the same hits
    and counts as the oracle)."""
    import torch
    base = scenes.gaussian_soup(3, seed=6)
    tris = np.tile(base, (400, 1))
    b, t, out = G.build(tris)
    w = mb.WideBVH.from_builder(b, t)
    v = base[0].reshape(3, 3).astype(np.float64)
    nrm = np.cross(v[1] - v[0], v[2] - v[1])
    nrm /= np.linalg.norm(nrm)
    rng = np.random.default_rng(3)
    rays = np.zeros((256, 8), np.float32)
    for i in range(len(rays)):
        d = np.cross(nrm, rng.standard_normal(3))
        d /= np.linalg.norm(d)
        rays[i, 0:3] = v.mean(0) + nrm * 1e-5 - d * 0.01
        rays[i, 4:7] = d
        rays[i, 7] = 0.02
    counts = torch.zeros(3 * len(rays), dtype=torch.int32, device="cuda")
    hits = G.host(mb.intersect_wide(w, G.dev(rays), counts=counts), np.uint32)
    c = G.host(counts, np.uint32).reshape(3, -1)
    ref, nv, nt, nr = O.trace_wide(O.build_wide(out["nodes"], len(tris)), out["nodes"], tris, out["root"], rays)
    np.testing.assert_array_equal(hits, ref)
    np.testing.assert_array_equal(c[2], nr)
    assert nr.sum() > 0


@pytest.mark.parametrize("quantised", [False, True])
def test_trace_wide_closest_matches_oracle(wcase, quantised):
    """Closest-hit rays over the FP32 and the quantised slots: the oracle's
    wide walk Hit records and counts exactly, and the stack-free walk's Hit
    records (on duplicated triangles, where copies give bit-identical t, the
    walk order picks which copy reports)."""
    import torch
    name, tris, b, t, out, w, rays = wcase
    if quantised:
        w.quantise()
    counts = torch.zeros(3 * len(rays), dtype=torch.int32, device="cuda")
    hits = G.host(mb.intersect_wide(w, G.dev(rays), counts=counts, quantised=quantised,
                                    rayQuery=mb.RAY_QUERY_CLOSEST), np.uint32)
    c = G.host(counts, np.uint32).reshape(3, -1)
    wide = O.build_wide(out["nodes"], len(tris))
    if quantised:
        q, _ = O.quantise_wide(wide, len(tris))
        ref, nv, nt, nr = O.trace_wide_quantised(q, out["nodes"], tris, out["root"], rays, query=0)
    else:
        ref, nv, nt, nr = O.trace_wide(wide, out["nodes"], tris, out["root"], rays, query=0)
    np.testing.assert_array_equal(hits, ref)
    np.testing.assert_array_equal(c[0], nv)
    np.testing.assert_array_equal(c[1], nt)
    np.testing.assert_array_equal(c[2], nr)
    plain = G.trace(b, t, rays, mb.RAY_QUERY_CLOSEST)
    if name == "duplicates":
        np.testing.assert_array_equal(hits[:, [0, 2, 3, 4, 5, 6]], plain[:, [0, 2, 3, 4, 5, 6]])
    else:
        np.testing.assert_array_equal(hits, plain)


def test_trace_wide_closest_restarts_on_stack_overflow(cuda):
    """400 nested copies of a triangle and rays parallel to their plane from
    outside the smallest ones: the closest-hit walk's stack overflows and the
    ray restarts with the stack-free walk (the oracle's hits and counts, the
    stack-free walk's hits), on FP32 and quantised slots."""
    import torch
    from test_oracle_walks import nested_triangles
    tris, rays = nested_triangles()
    b, t, out = G.build(tris)
    w = mb.WideBVH.from_builder(b, t).quantise()
    wide = O.build_wide(out["nodes"], len(tris))
    plain = G.trace(b, t, rays, mb.RAY_QUERY_CLOSEST)
    for quantised in (False, True):
        counts = torch.zeros(3 * len(rays), dtype=torch.int32, device="cuda")
        hits = G.host(mb.intersect_wide(w, G.dev(rays), counts=counts, quantised=quantised,
                                        rayQuery=mb.RAY_QUERY_CLOSEST), np.uint32)
        c = G.host(counts, np.uint32).reshape(3, -1)
        if quantised:
            ref, nv, nt, nr = O.trace_wide_quantised(O.quantise_wide(wide, len(tris))[0], out["nodes"], tris,
                                                     out["root"], rays, query=0)
        else:
            ref, nv, nt, nr = O.trace_wide(wide, out["nodes"], tris, out["root"], rays, query=0)
        np.testing.assert_array_equal(hits, ref)
        np.testing.assert_array_equal(c, np.stack([nv, nt, nr]))
        np.testing.assert_array_equal(hits, plain)
        assert nr.sum() > 0


def _ao(fn, w, h, ns, radius, sobol, *args):
    import torch
    px = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    occ = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    stats = torch.zeros(8, dtype=torch.int64, device="cuda")
    fn(px, (w, h), *args, sobol, ns, radius, 12345, occluded=occ, stats=stats)
    torch.cuda.synchronize()
    st = G.host(stats)
    return G.host(px, np.uint32), G.host(occ, np.uint32), st


@pytest.mark.parametrize("sobol", [1, 0])
def test_ao_wide_equals_plain_heightfield(cuda, sobol):
    """212,992-triangle heightfield + icospheres, 512 x 512, 16 AO rays of
    radius 0.25: every occlusion count and pixel of the plain form."""
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = mb.RayGenerator.from_array(O.lookat(eye, c, up, fovy, 512, 512))
    px0, occ0, st0 = _ao(lambda *a, **k: mb.render_ao(a[0], a[1], a[2], b.m_rootNode, b.m_internals, t, *a[3:], **k),
                         512, 512, 16, 0.25, sobol, cam)
    w = mb.WideBVH.from_builder(b, t)
    px1, occ1, st1 = _ao(mb.render_ao_wide, 512, 512, 16, 0.25, sobol, cam, w)
    np.testing.assert_array_equal(occ1, occ0)
    np.testing.assert_array_equal(px1, px0)
    assert st1[0] == st0[0]          # the same rays
    assert st1[3] < 0.5 * st0[3]     # AO-ray node visits: wide nodes, fewer than half the stack-free walk's
    assert st1[6] == 0               # no restarts on this scene


def test_quantised_wide_slots_match_oracle(wcase):
    import torch
    _, tris, _, _, out, w, _ = wcase
    n = len(tris)
    w.quantise()
    torch.cuda.synchronize()
    assert int(G.host(w.status)[0]) == 0
    if n == 1:
        return
    got = G.host(w.qwide, np.uint32)[: n - 1]
    ref, ok = O.quantise_wide(O.build_wide(out["nodes"], n), n)
    assert ok
    bad = np.nonzero((got != ref).any(1))[0]
    assert bad.size == 0, f"{bad.size} slots differ, first {bad[:4]}: {got[bad[:1]]} vs {ref[bad[:1]]}"


def test_trace_wide_quantised_matches_oracle(wcase):
    import torch
    name, tris, b, t, out, w, rays = wcase
    w.quantise()
    counts = torch.zeros(3 * len(rays), dtype=torch.int32, device="cuda")
    hits = G.host(mb.intersect_wide(w, G.dev(rays), counts=counts, quantised=True), np.uint32)
    c = G.host(counts, np.uint32).reshape(3, -1)
    q, _ = O.quantise_wide(O.build_wide(out["nodes"], len(tris)), len(tris))
    ref, nv, nt, nr = O.trace_wide_quantised(q, out["nodes"], tris, out["root"], rays)
    np.testing.assert_array_equal(hits, ref)
    np.testing.assert_array_equal(c[0], nv)
    np.testing.assert_array_equal(c[1], nt)
    np.testing.assert_array_equal(c[2], nr)
    plain = G.trace(b, t, rays, mb.RAY_QUERY_ANY)
    np.testing.assert_array_equal(hits[:, 7] == MISS, plain[:, 7] == MISS)


def test_quantised_wide_fallback_on_huge_extents(cuda):
    """Coordinates spread over about 1e37 cannot be quantised: the status
    word is set and every ray takes the stack-free walk (the oracle's hits)."""
    rng = np.random.default_rng(9)
    tris = (rng.random((200, 9)).astype(np.float32) - np.float32(0.5)) * np.float32(2e37)
    b, t, out = G.build(tris)
    w = mb.WideBVH.from_builder(b, t).quantise()
    rays = scenes.random_rays(500, [-1e37, -1e37, -1e37], [1e37, 1e37, 1e37], seed=2)
    rays[:, 7] = np.float32(3e37)
    hits = G.host(mb.intersect_wide(w, G.dev(rays), quantised=True), np.uint32)
    assert int(G.host(w.status)[0]) == 1
    ref = O.trace(out["nodes"], tris, out["root"], rays, 1, 0)
    np.testing.assert_array_equal(hits, ref)


@pytest.mark.parametrize("sobol", [1, 0])
def test_ao_quantised_wide_equals_plain_heightfield(cuda, sobol):
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = mb.RayGenerator.from_array(O.lookat(eye, c, up, fovy, 512, 512))
    px0, occ0, st0 = _ao(lambda *a, **k: mb.render_ao(a[0], a[1], a[2], b.m_rootNode, b.m_internals, t, *a[3:], **k),
                         512, 512, 16, 0.25, sobol, cam)
    w = mb.WideBVH.from_builder(b, t).quantise()
    px1, occ1, st1 = _ao(lambda *a, **k: mb.render_ao_wide(*a, quantised=True, **k), 512, 512, 16, 0.25, sobol, cam,
                         w)
    np.testing.assert_array_equal(occ1, occ0)
    np.testing.assert_array_equal(px1, px0)
    assert st1[0] == st0[0] and st1[3] < 0.5 * st0[3]
