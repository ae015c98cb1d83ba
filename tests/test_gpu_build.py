"""GPU build parity: sorted keys, permutation, deltas, every InternalNode
word and the root must equal the oracle's bit for bit (the oracle is pinned
to the reference's own BVHCPUBuilder with a stable key order)."""
import os

import numpy as np
import pytest

import _gpu as G
import _oracle as O
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", ["soup1", "soup2", "soup3", "soup257", "soup4097", "dup300", "small_scene",
                                  "normal1000"])
def test_build_matches_golden(cuda, case):
    g = np.load(os.path.join(GOLD, "builds.npz"))
    tris = g[f"{case}/tris"]
    _, _, out = G.build(tris, int(g[f"{case}/option"][0]))
    ref = {k: g[f"{case}/{k}"] for k in ("nodes", "deltas", "keys", "indices", "scene")}
    ref["root"] = int(g[f"{case}/root"][0])
    G.assert_build_equal(out, ref)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 31, 32, 33, 255, 256, 257, 4095, 4096, 4097, 8191, 8193, 65537, 300001])
def test_build_sizes(cuda, n):
    tris = scenes.gaussian_soup(n, clusters=8, seed=1000 + n)
    _, _, out = G.build(tris)
    G.assert_build_equal(out, O.build(tris))


def test_build_heightfield_scene(cuda):
    tris = scenes.heightfield_icospheres()
    _, _, out = G.build(tris)
    G.assert_build_equal(out, O.build(tris))


@pytest.mark.parametrize("kind", ["all_equal", "two_values", "axis_aligned_zero"])
def test_build_duplicate_keys(cuda, kind):
    base = scenes.gaussian_soup(2, seed=77)
    if kind == "all_equal":
        tris = np.tile(base[:1], (5000, 1))
    elif kind == "two_values":
        tris = np.tile(base, (20000, 1))
    else:
        # a flat sheet in z = 0 (+0 and -0 coordinates) with a degenerate axis
        rng = np.random.default_rng(5)
        p = rng.random((3000, 3, 3)).astype(np.float32)
        p[..., 2] = np.where(rng.random((3000, 3)) < 0.5, np.float32(0.0), np.float32(-0.0))
        tris = p.reshape(-1, 9)
    _, _, out = G.build(tris)
    G.assert_build_equal(out, O.build(tris))


def test_build_use_normal_option(cuda):
    tris = scenes.gaussian_soup(50000, clusters=4, seed=3)
    _, _, out = G.build(tris, 1)
    G.assert_build_equal(out, O.build(tris, 1))


def test_build_reuses_scratch_across_sizes(cuda):
    import minimumlbvh_b200 as mb
    sorter = mb.OnesweepSort()
    for n in (70000, 1000, 70000, 3):
        tris = scenes.gaussian_soup(n, clusters=3, seed=n)
        _, _, out = G.build(tris, 0, sorter)
        G.assert_build_equal(out, O.build(tris))


def test_build_on_side_stream(cuda):
    import torch
    s = torch.cuda.Stream()
    tris = scenes.gaussian_soup(100000, seed=8)
    with torch.cuda.stream(s):
        _, _, out = G.build(tris, 0, None, s)
    G.assert_build_equal(out, O.build(tris))


def test_build_full_size_soup(cuda):
    """The 4,194,304-triangle Gaussian soup: bit-exact against the oracle and
    structurally valid (every leaf once, parents, containment, delta order)."""
    tris = scenes.gaussian_soup()
    b, t, out = G.build(tris)
    ref = O.build(tris)
    G.assert_build_equal(out, ref)
    n = len(tris)
    assert (np.diff(out["keys"].astype(np.int64)) >= 0).all()
    assert np.array_equal(np.sort(out["indices"]), np.arange(n, dtype=np.uint32))
    L = O.oracle()
    assert L.orc_check_tree(O.P(out["nodes"]), O.P(tris), n, out["root"]) == 1
    assert L.orc_validate(O.P(out["nodes"]), O.P(out["deltas"]), n, out["root"], 255) == 1
