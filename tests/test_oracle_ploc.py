"""The higher-quality (PLOC) build on the oracle (CPU only).

The reference's higher-quality build is Embree's SAH builder behind
BVHCPUBuilder::buildByEmbree (minimum_lbvh.h:594-656), a binary-only
dependency: its trees cannot be reproduced here. What the reference fixes is
the output form, one triangle per leaf in the InternalNode array that every
walk reads, and that is what these tests hold the oracle's PLOC tree to:
a valid tree (every triangle once, exact leaf boxes, parent links), nodes in
in-order with build_lbvh's context convention (the escape index of
intersect_escape_link), every walk of the reference (its own compiled code
where it is built) answering the same closest distances and any-hit
verdicts as on the LBVH, and a smaller surface-area cost than the LBVH."""
import numpy as np
import pytest

import _oracle as O
from minimumlbvh_b200 import scenes

LEAF = 0x80000000
INVALID = 0x7FFFFFFF


def _scenes():
    yield "soup", scenes.gaussian_soup(20000, clusters=8, seed=5), ([0, 0, 0], [1, 1, 1])
    yield "heightfield", scenes.heightfield_icospheres(quads=64, spheres=8), ([-1, -0.3, -1], [1, 0.7, 1])
    dup = np.tile(scenes.gaussian_soup(3, seed=6), (400, 1))  # equal boxes everywhere: ties at every step
    yield "duplicates", dup, ([0, 0, 0], [1, 1, 1])


@pytest.fixture(scope="module", params=["soup", "heightfield", "duplicates"])
def case(request):
    for name, tris, box in _scenes():
        if name == request.param:
            lb = O.build(tris)
            pl = O.build_ploc(tris, 0, 8)
            rays = scenes.random_rays(6000, box[0], box[1], seed=13)
            rays[1::3, 7] = 0.05  # short rays, as AO rays are
            return name, tris, lb, pl, rays


def in_order(nodes, root, n):
    """Leaves and internal nodes of a left-to-right walk, interleaved."""
    seq, stack, node = [], [], root
    while stack or node is not None:
        while node is not None and not (node & LEAF):
            stack.append(node)
            node = int(nodes[node, 0])
        if node is not None:
            seq.append(("leaf", node & ~LEAF))
            node = None
        if stack:
            p = stack.pop()
            seq.append(("node", p))
            node = int(nodes[p, 1])
    return seq


def escape(nodes, root, x):
    cur = x
    while cur != root:
        p = int(nodes[cur, 14])
        if int(nodes[p, 0]) == cur:
            return p
        cur = p
    return 0xFFFFFFFF


def test_tree_is_valid(case):
    _, tris, _, pl, _ = case
    assert O.check_tree(pl["nodes"], tris, pl["root"])
    assert int(pl["nodes"][pl["root"], 14]) == INVALID


def test_nodes_in_in_order_with_escape_context(case):
    _, tris, _, pl, _ = case
    n = len(tris)
    seq = in_order(pl["nodes"], pl["root"], n)
    assert [k for k, _ in seq] == ["leaf", "node"] * (n - 1) + ["leaf"]
    assert [v for k, v in seq if k == "node"] == list(range(n - 1))
    rng = np.random.default_rng(1)
    for x in rng.integers(0, n - 1, 300):
        assert int(pl["nodes"][x, 15]) == escape(pl["nodes"], pl["root"], int(x))


def test_smaller_surface_area_cost(case):
    name, _, lb, pl, _ = case
    if name == "duplicates":
        pytest.skip("every box is one of three: no tree is better")
    assert O.sah_cost(pl["nodes"], pl["root"]) < 0.95 * O.sah_cost(lb["nodes"], lb["root"])


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_closest_hits_as_on_the_lbvh(case, mode):
    """Stack-free, escape-link and stackful walks over the PLOC tree find the
    same closest distance (and hit/miss) as over the LBVH; the triangle may
    differ only where two triangles meet the ray at the same distance."""
    name, tris, lb, pl, rays = case
    a = O.trace(lb["nodes"], tris, lb["root"], rays, 0, 0)
    b = O.trace(pl["nodes"], tris, pl["root"], rays, 0, mode)
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    same = a[:, 7] == b[:, 7]
    if name != "duplicates":
        assert same.mean() > 0.999
    np.testing.assert_array_equal(a[same][:, [2, 3, 4, 5, 6]], b[same][:, [2, 3, 4, 5, 6]])


def test_any_hit_as_on_the_lbvh(case):
    _, tris, lb, pl, rays = case
    a = O.trace(lb["nodes"], tris, lb["root"], rays, 1, 0)
    b = O.trace(pl["nodes"], tris, pl["root"], rays, 1, 0)
    np.testing.assert_array_equal(a[:, 7] != 0xFFFFFFFF, b[:, 7] != 0xFFFFFFFF)


def test_replay_and_wide_walks_take_the_tree(case):
    _, tris, _, pl, rays = case
    n = len(tris)
    sf = O.trace(pl["nodes"], tris, pl["root"], rays, 0, 0)
    rp = O.trace_replay(pl["nodes"], tris, pl["root"], rays, 0, 16)
    np.testing.assert_array_equal(sf, rp)
    anyh = O.trace(pl["nodes"], tris, pl["root"], rays, 1, 0)
    wide = O.build_wide(pl["nodes"], n)
    wh = O.trace_wide(wide, pl["nodes"], tris, pl["root"], rays)[0]
    np.testing.assert_array_equal(anyh[:, 7] != 0xFFFFFFFF, wh[:, 7] != 0xFFFFFFFF)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reference_walks_over_the_tree(case, mode):
    """The reference's own intersect_stackfree / intersect_escape_link /
    intersect_stackfull (compiled from its sources) over the PLOC tree return
    the oracle's Hit records."""
    _, tris, _, pl, rays = case
    for query in (0, 1) if mode != 2 else (0,):
        exp = O.trace(pl["nodes"], tris, pl["root"], rays, query, mode)
        got = O.ref_trace(pl["nodes"], tris, pl["root"], rays, query, mode)
        cols = [0, 2, 3, 4, 5, 6, 7]
        np.testing.assert_array_equal(got[:, cols], exp[:, cols])


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 17, 1023, 1024, 1025, 2049])
@pytest.mark.parametrize("radius", [1, 8, 32])
def test_sizes_and_radii(n, radius):
    tris = scenes.gaussian_soup(n, clusters=4, seed=n)
    pl = O.build_ploc(tris, 0, radius)
    if n == 1:
        assert pl["root"] == LEAF
        return
    assert O.check_tree(pl["nodes"], tris, pl["root"])
    seq = in_order(pl["nodes"], pl["root"], n)
    assert [v for k, v in seq if k == "node"] == list(range(n - 1))


def test_normal_option_and_nan():
    tris = scenes.gaussian_soup(3000, clusters=4, seed=9)
    pl = O.build_ploc(tris, 1, 8)
    assert O.check_tree(pl["nodes"], tris, pl["root"])
    bad = tris.copy()
    bad[::97, 4] = np.nan  # NaN boxes sort above every area: the build still ends with one root
    pl = O.build_ploc(bad, 0, 8)
    seq = in_order(pl["nodes"], pl["root"], len(bad))
    assert sorted(v for k, v in seq if k == "leaf") == list(range(len(bad)))


def test_bad_arguments():
    tris = scenes.gaussian_soup(10, seed=1)
    nodes = np.zeros((9, 16), np.uint32)
    root = np.zeros(1, np.uint32)
    assert O.oracle().orc_build_ploc(O.P(tris), 10, 0, 0, O.P(nodes), O.P(root)) < 0
    assert O.oracle().orc_build_ploc(O.P(tris), 0, 0, 8, O.P(nodes), O.P(root)) < 0


@pytest.mark.parametrize("kind", ["identical", "collinear", "chain"])
def test_stalls_end_in_few_iterations(kind):
    """Inputs where ties (identical boxes, zero union areas) or a chain of
    growing gaps let only one pair merge per run and iteration: the stall
    rules keep the iteration count logarithmic (it would be about n without
    them)."""
    n = 20000
    if kind == "identical":
        tris = np.tile(scenes.gaussian_soup(1, seed=4), (n, 1))
    elif kind == "collinear":
        x = np.sort(np.random.default_rng(3).random(n)).astype(np.float32)
        tris = np.zeros((n, 9), np.float32)
        tris[:, 0], tris[:, 3], tris[:, 6] = x, x + 0.001, x + 0.002
    else:
        x = np.cumsum(1.0 + np.arange(n) * 1e-3)
        x = (x / x[-1]).astype(np.float32)
        tris = np.zeros((n, 9), np.float32)
        tris[:, 0], tris[:, 3], tris[:, 4] = x, x + 1e-6, 0.001
        tris[:, 6], tris[:, 7], tris[:, 8] = x, 0.001, 0.0005
    pl = O.build_ploc(np.ascontiguousarray(tris, np.float32), 0, 8)
    assert O.check_tree(pl["nodes"], tris, pl["root"])
    assert pl["iterations"] < 150
