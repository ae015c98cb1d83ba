"""The replay walk and the quantised form on the oracle (CPU only). The
replay walk over the reference node layout returns intersect_stackfree's Hit
records bit for bit at every stack depth. Decoded quantised child boxes contain
the FP32 boxes, the quantised stack-free walk returns the FP32 tree's closest
hits, and the replay walk (a stack of pending far children instead of
revisits, with the stack-free walk taking over when the stack is full)
returns the stack-free walk's Hit records bit for bit at every stack depth,
with fewer node visits."""
import numpy as np
import pytest

import _oracle as O
from minimumlbvh_b200 import scenes


def _scenes():
    yield "soup", scenes.gaussian_soup(20000, clusters=8, seed=5), ([0, 0, 0], [1, 1, 1])
    yield "heightfield", scenes.heightfield_icospheres(quads=64, spheres=8), ([-1, -0.3, -1], [1, 0.7, 1])
    dup = np.tile(scenes.gaussian_soup(3, seed=6), (400, 1))  # long chains of equal keys: deep trees
    yield "duplicates", dup, ([0, 0, 0], [1, 1, 1])


@pytest.fixture(scope="module", params=["soup", "heightfield", "duplicates"])
def case(request):
    for name, tris, box in _scenes():
        if name == request.param:
            b = O.build(tris)
            q = O.quantise(b, tris)
            rays = scenes.random_rays(6000, box[0], box[1], seed=13)
            rays[1::3, 7] = 0.05  # short rays, as AO rays are
            return name, tris, b, q, rays


def test_quantised_boxes_contain_fp32_boxes(case):
    _, tris, b, q, _ = case
    assert O.oracle().orc_check_quantised(O.P(b["nodes"]), len(tris), O.P(q["qnodes"]), O.P(q["header"])) == 1


def test_quantised_walk_finds_fp32_closest_hits(case):
    _, tris, b, q, rays = case
    got = O.trace_quantised(q, rays, 0)
    plain = O.trace(b["nodes"], tris, b["root"], rays, 0, 0)
    np.testing.assert_array_equal(got[:, 7], plain[:, 7])
    np.testing.assert_array_equal(got[:, 0], plain[:, 0])


@pytest.mark.parametrize("query", [0, 1])
@pytest.mark.parametrize("depth", [1, 2, 3, 8, 16, 64])
def test_replay_walk_equals_stackfree_walk(case, query, depth):
    name, _, _, q, rays = case
    ref, nv0, nt0, nu0 = O.trace_quantised(q, rays, query, counters=True)
    got, nv1, nt1, nu1 = O.trace_quantised(q, rays, query, counters=True, stack_depth=depth)
    np.testing.assert_array_equal(got, ref)
    # the same leaves in the same order, fewer internal-node visits
    np.testing.assert_array_equal(nt1, nt0)
    assert (nv1 <= nv0).all()
    if depth >= 16 and query == 0 and name != "duplicates":  # deep chains overflow the stack
        assert nv1.sum() < 0.75 * nv0.sum()


@pytest.mark.parametrize("query", [0, 1])
@pytest.mark.parametrize("depth", [1, 2, 5, 16, 64])
def test_replay_walk_equals_stackfree_on_fp32_nodes(case, query, depth):
    name, tris, b, _, rays = case
    ref, nv0, nt0 = O.trace(b["nodes"], tris, b["root"], rays, query, 0, counters=True)
    got, nv1, nt1 = O.trace_replay(b["nodes"], tris, b["root"], rays, query, depth, counters=True)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(nt1, nt0)  # the same leaves, in the same order
    assert (nv1 <= nv0).all()
    if depth >= 16 and query == 0 and name != "duplicates":
        assert nv1.sum() < 0.75 * nv0.sum()


def test_fp32_hit_distances_within_fp64_bound(case):
    """Every closest hit's FP32 t is within the stated forward error bound of
    the FP64 evaluation of the same ray-plane formula (fp64check)."""
    from minimumlbvh_b200 import fp64check as F
    name, tris, b, q, rays = case
    hits = O.trace(b["nodes"], tris, b["root"], rays, 0, 0)
    r = F.check_hits(tris, rays, hits)
    assert (r["hits"] > 0 or name == "duplicates") and r["max_bound_ratio"] <= 1.0, r
    rq = F.check_hits(tris, rays, O.trace_quantised(q, rays, 0))
    assert rq == r
