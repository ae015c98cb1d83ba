"""GPU parity of the higher-quality build (mlbvh_build_ploc; the reference's
counterpart is Embree's SAH build behind BVHCPUBuilder::buildByEmbree,
minimum_lbvh.h:594-656, which cannot run here). Every node word and the root
must equal the oracle's PLOC restatement bit for bit: sizes on both sides of
the shared-memory tail (1,024 clusters) and of a 1,024-cluster tile, radii
1-32, the normal-key option, equal boxes everywhere, the 212,992-triangle
heightfield and the 4M-triangle soup. Over the GPU's tree, every walk and
shading entry point answers what the oracle answers over the same tree."""
import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF
HIT_COLS = [0, 2, 3, 4, 5, 6, 7]  # the Hit padding word is not written


def gpu_ploc(tris, option=0, radius=8, sorter=None):
    import torch
    t = G.dev(np.ascontiguousarray(tris, np.float32).reshape(-1, 9))
    n = len(tris)
    b = mb.BVHGPUBuilder().buildByPLOC(t, n, option, sorter, radius)
    b.status()
    torch.cuda.synchronize()
    out = dict(nodes=G.host(b.m_internals, np.uint32)[: n - 1], root=int(G.host(b.m_rootNode, np.uint32)[0]))
    if n > 1:
        assert O.check_tree(out["nodes"], tris, out["root"]), "GPU PLOC build produced an invalid tree"
    return b, t, out


def assert_same_tree(got, ref, n):
    assert got["root"] == ref["root"], (got["root"], ref["root"])
    if n > 1:
        bad = np.nonzero((got["nodes"] != ref["nodes"]).any(1))[0]
        assert bad.size == 0, f"{bad.size} nodes differ, first {bad[:5]}"


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 1023, 1024, 1025, 2049, 5000, 65537])
@pytest.mark.parametrize("radius", [1, 8, 32])
def test_ploc_matches_oracle_sizes(cuda, n, radius):
    tris = scenes.gaussian_soup(n, clusters=4, seed=n)
    _, _, got = gpu_ploc(tris, 0, radius)
    assert_same_tree(got, O.build_ploc(tris, 0, radius), n)


@pytest.mark.parametrize("name", ["heightfield", "duplicates", "normal_keys"])
def test_ploc_matches_oracle_scenes(cuda, name):
    option = 0
    if name == "heightfield":
        tris = scenes.heightfield_icospheres()
    elif name == "duplicates":
        tris = np.tile(scenes.gaussian_soup(3, seed=6), (4000, 1))
    else:
        tris, option = scenes.gaussian_soup(40000, clusters=8, seed=4), 1
    t = G.dev(tris)
    b = mb.BVHGPUBuilder().buildByPLOC(t, len(tris), option, None, 8)
    b.status()
    got = dict(nodes=G.host(b.m_internals, np.uint32)[: len(tris) - 1],
               root=int(G.host(b.m_rootNode, np.uint32)[0]))
    assert_same_tree(got, O.build_ploc(tris, option, 8), len(tris))


def test_ploc_nan_vertices_end_with_one_tree(cuda):
    """NaN vertices: the Morton key of a NaN centroid is a float-to-integer
    conversion of NaN, which the reference leaves to the platform (CPU and GPU
    differ), so the tree is not pinned; the build must still end (NaN areas
    order above all others) with every triangle once and in-order nodes."""
    tris = scenes.gaussian_soup(20000, clusters=8, seed=8)
    tris[::97, 4] = np.nan
    t = G.dev(tris)
    n = len(tris)
    b = mb.BVHGPUBuilder().buildByPLOC(t, n, 0, None, 8)
    b.status()
    nodes = G.host(b.m_internals, np.uint32)[: n - 1]
    root = int(G.host(b.m_rootNode, np.uint32)[0])
    assert int(nodes[root, 14]) == 0x7FFFFFFF
    leaves, inner, stack, node = [], [], [], root
    while stack or node is not None:
        while node is not None and not (node & 0x80000000):
            stack.append(node)
            node = int(nodes[node, 0])
        if node is not None:
            leaves.append(node & 0x7FFFFFFF)
            node = None
        if stack:
            p = stack.pop()
            inner.append(p)
            node = int(nodes[p, 1])
    assert sorted(leaves) == list(range(n))
    assert inner == list(range(n - 1))


def test_ploc_matches_oracle_soup4m(cuda):
    """4,194,304-triangle Gaussian soup, radius 8 (the bench's workload)."""
    tris = scenes.gaussian_soup()
    _, _, got = gpu_ploc(tris, 0, 8)
    ref = O.build_ploc(tris, 0, 8)
    assert_same_tree(got, ref, len(tris))
    lb = O.build(tris)
    assert O.sah_cost(got["nodes"], got["root"]) < 0.92 * O.sah_cost(lb["nodes"], lb["root"])


def test_ploc_scratch_shared_with_lbvh_builds(cuda):
    """One sorter (scratch) for LBVH and PLOC builds in turn: each output as
    if alone, and repeated PLOC builds identical."""
    tris = scenes.gaussian_soup(30000, clusters=8, seed=12)
    sorter = mb.OnesweepSort(0)
    ref = O.build_ploc(tris, 0, 8)
    _, _, a = gpu_ploc(tris, 0, 8, sorter)
    b, t, lb = G.build(tris, sorter=sorter)
    G.assert_build_equal(lb, O.build(tris))
    _, _, c = gpu_ploc(tris, 0, 8, sorter)
    assert_same_tree(a, ref, len(tris))
    assert_same_tree(c, ref, len(tris))


@pytest.fixture(scope="module")
def ploc_case(cuda):
    tris = scenes.heightfield_icospheres()
    b, t, out = gpu_ploc(tris, 0, 8)
    rays = scenes.random_rays(30000, [-1, -0.3, -1], [1, 0.7, 1], seed=21)
    rays[1::3, 7] = 0.05
    return tris, b, t, out, rays


@pytest.mark.parametrize("query", [0, 1])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_walks_over_ploc_tree(ploc_case, query, mode):
    """Stack-free, escape-link, stackful and replay walks over the GPU's PLOC
    tree return the oracle's Hit records over the same tree."""
    tris, b, t, out, rays = ploc_case
    if mode == 2 and query == 1:
        pytest.skip("the stackful walk answers closest hits only")
    got = G.trace(b, t, rays, query, mode)
    ref = O.trace(out["nodes"], tris, out["root"], rays, query, 0 if mode == 3 else mode)
    np.testing.assert_array_equal(got[:, HIT_COLS], ref[:, HIT_COLS])


def test_ao_over_ploc_tree(ploc_case):
    """AO (512 x 512, 16 rays of radius 0.25) over the PLOC tree: the
    oracle's occlusion counts over that tree for the plain, replay and 4-wide
    forms (FP32 and quantised), and every count equal to the LBVH's."""
    import torch
    tris, b, t, out, _ = ploc_case
    eye, c, up, fovy = scenes.camera_heightfield()
    w = h = 512
    cam_arr = O.lookat(eye, c, up, fovy, w, h)
    cam = mb.RayGenerator.from_array(cam_arr)
    _, rocc = O.render_ao(cam_arr, out["root"], out["nodes"], tris, w, h, 16, 0.25, 12345, 1, trig=1)

    def run(fn):
        px = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        occ = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        fn(px, occ)
        torch.cuda.synchronize()
        return G.host(occ, np.uint32)

    lt = mb.leaf_triangles(b, t)
    wide = mb.WideBVH.from_builder(b, t)
    wide.quantise()
    forms = {
        "plain": lambda px, occ: mb.render_ao(px, (w, h), cam, b.m_rootNode, b.m_internals, t, 1, 16, 0.25, 12345,
                                              occluded=occ),
        "replay": lambda px, occ: mb.render_ao(px, (w, h), cam, b.m_rootNode, b.m_internals, t, 1, 16, 0.25, 12345,
                                               occluded=occ, traversal=mb.TRAVERSAL_REPLAY, leaf_triangles=lt),
        "wide": lambda px, occ: mb.render_ao_wide(px, (w, h), cam, wide, 1, 16, 0.25, 12345, occluded=occ),
        "wide_quantised": lambda px, occ: mb.render_ao_wide(px, (w, h), cam, wide, 1, 16, 0.25, 12345, occluded=occ,
                                                            quantised=True),
    }
    for name, fn in forms.items():
        np.testing.assert_array_equal(run(fn), rocc, err_msg=name)
    lb = O.build(tris)
    _, locc = O.render_ao(cam_arr, lb["root"], lb["nodes"], tris, w, h, 16, 0.25, 12345, 1, trig=1)
    np.testing.assert_array_equal(rocc, locc)


def test_quantised_tree_over_ploc_tree(ploc_case):
    """The binary quantised tree made from the PLOC tree: the oracle's
    quantised Hit records over that tree."""
    tris, b, t, out, rays = ploc_case
    q = mb.QuantisedBVH.from_builder(b, t)
    got = G.host(mb.intersect_quantised(q, G.dev(rays)), np.uint32)
    ref = O.trace_quantised(O.quantise(out, tris), rays)
    np.testing.assert_array_equal(got[:, HIT_COLS], ref[:, HIT_COLS])


def test_ploc_build_captures_in_a_graph(cuda):
    """The whole PLOC build (key and sort passes, k_ploc_init, the cooperative
    k_ploc) captured in a CUDA graph on a side stream: the replay writes the
    oracle's tree."""
    import torch
    tris = scenes.gaussian_soup(200000, clusters=8, seed=3)
    n = len(tris)
    t = G.dev(tris)
    b = mb.BVHGPUBuilder()
    s = mb.OnesweepSort(0)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        b.buildByPLOC(t, n, 0, s, 8, stream=st)  # allocations outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        b.buildByPLOC(t, n, 0, s, 8, stream=st)
    b.m_internals.zero_()
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    b.status()
    got = dict(nodes=G.host(b.m_internals, np.uint32)[: n - 1], root=int(G.host(b.m_rootNode, np.uint32)[0]))
    assert_same_tree(got, O.build_ploc(tris, 0, 8), n)


@pytest.mark.parametrize("radius,n", [(8, 1008), (8, 1009), (8, 2016), (8, 2017), (32, 960), (32, 961), (32, 1921),
                                      (1, 1022), (1, 1023), (16, 992), (16, 993), (4, 1016), (4, 1025)])
def test_ploc_tile_boundaries(cuda, radius, n):
    """Cluster counts at the edges of a tile (kTile - 2r clusters) and of the
    single-CTA tail (1,024 clusters)."""
    tris = scenes.gaussian_soup(n, clusters=3, seed=n + radius)
    _, _, got = gpu_ploc(tris, 0, radius)
    assert_same_tree(got, O.build_ploc(tris, 0, radius), n)


def chain_triangles(n):
    """Thin triangles along x with strictly growing gaps: each cluster's
    nearest neighbour is the one before it, PLOC's worst case without ties."""
    x = np.cumsum(1.0 + np.arange(n) * 1e-3)
    x = (x / x[-1]).astype(np.float32)
    tris = np.zeros((n, 9), np.float32)
    tris[:, 0] = x
    tris[:, 3] = x + 1e-6
    tris[:, 4] = 0.001
    tris[:, 6] = x
    tris[:, 7] = 0.001
    tris[:, 8] = 0.0005
    return tris


@pytest.mark.parametrize("kind", ["identical", "points", "collinear", "chain"])
def test_ploc_degenerate_inputs(cuda, kind):
    """Every area key equal (one triangle repeated), zero-area triangles at a
    few points, triangles along a line, and a chain of growing gaps: the
    stall rules (hashed ties, then a pairing iteration) take the same turns
    on both sides, and the tree is the oracle's."""
    rng = np.random.default_rng(17)
    n = 20000 if kind == "chain" else 5000
    if kind == "chain":
        tris = chain_triangles(n)
    elif kind == "identical":
        tris = np.tile(scenes.gaussian_soup(1, seed=4), (n, 1))
    elif kind == "points":
        pts = rng.random((7, 3)).astype(np.float32)
        tris = np.repeat(pts[rng.integers(0, 7, n)], 3, axis=0).reshape(n, 9)
    else:
        x = np.sort(rng.random(n)).astype(np.float32)
        tris = np.zeros((n, 9), np.float32)
        tris[:, 0] = x
        tris[:, 3] = x + 0.001
        tris[:, 6] = x + 0.002
    tris = np.ascontiguousarray(tris, np.float32)
    t = G.dev(tris)
    b = mb.BVHGPUBuilder().buildByPLOC(t, n, 0, None, 8)
    b.status()
    got = dict(nodes=G.host(b.m_internals, np.uint32)[: n - 1], root=int(G.host(b.m_rootNode, np.uint32)[0]))
    ref = O.build_ploc(tris, 0, 8)
    assert_same_tree(got, ref, n)
    assert O.check_tree(ref["nodes"], tris, ref["root"])
