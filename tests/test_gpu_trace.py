"""GPU query parity: every Hit word (t, uv, ng, triangle index) of the
stack-free, escape-link and stackful traversals must equal the oracle's
(pinned to the reference's intersect_* functions) bit for bit, and the replay
walk (mode 3) must give the stack-free walk's Hit records."""
import os

import numpy as np
import pytest

import _gpu as G
import _oracle as O
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
COMBOS = [(0, 0), (1, 0), (0, 1), (1, 1), (0, 2)]
ALL = COMBOS + [(0, 3), (1, 3)]  # mode 3: the replay walk (the oracle restates it too)


@pytest.mark.parametrize("q,m", COMBOS)
def test_trace_matches_golden(cuda, q, m):
    g = np.load(os.path.join(GOLD, "builds.npz"))
    tris = g["small_scene/tris"]
    b, t, _ = G.build(tris)
    tr = np.load(os.path.join(GOLD, "traces.npz"))
    np.testing.assert_array_equal(G.trace(b, t, tr["rays"], q, m), tr[f"hits_q{q}_m{m}"])
    np.testing.assert_array_equal(G.trace(b, t, tr["short_rays"], q, m), tr[f"short_q{q}_m{m}"])
    if m == 0:  # the replay walk reproduces the reference's stack-free hits
        np.testing.assert_array_equal(G.trace(b, t, tr["rays"], q, 3), tr[f"hits_q{q}_m0"])
        np.testing.assert_array_equal(G.trace(b, t, tr["short_rays"], q, 3), tr[f"short_q{q}_m0"])


@pytest.fixture(scope="module")
def heightfield(cuda):
    tris = scenes.heightfield_icospheres()
    b, t, out = G.build(tris)
    return tris, b, t, out


@pytest.mark.parametrize("q,m", ALL)
def test_trace_heightfield(heightfield, q, m):
    tris, b, t, out = heightfield
    rays = scenes.random_rays(200000, [-1, -0.3, -1], [1, 0.7, 1], seed=21)
    rays[1::3, 7] = 0.25  # AO-length rays
    got = G.trace(b, t, rays, q, m)
    exp = O.trace(out["nodes"], tris, out["root"], rays, q, m)
    np.testing.assert_array_equal(got, exp)
    assert (got[:, 7] != 0xFFFFFFFF).mean() > 0.2


def test_trace_axis_parallel_rays(heightfield):
    """Direction components of exactly 0 exercise invRd's clamp to +-FLT_MAX."""
    tris, b, t, out = heightfield
    rng = np.random.default_rng(4)
    n = 30000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform([-1.1, -0.3, -1.1], [1.1, 0.8, 1.1], (n, 3))
    axis = rng.integers(0, 3, n)
    rays[np.arange(n), 4 + axis] = np.where(rng.random(n) < 0.5, 1.0, -1.0)
    rays[::5, 4:7] = np.where(rays[::5, 4:7] == 0, np.float32(-0.0), rays[::5, 4:7])
    rays[:, 7] = O.FLT_MAX
    for q, m in ALL:
        np.testing.assert_array_equal(G.trace(b, t, rays, q, m), O.trace(out["nodes"], tris, out["root"], rays, q, m))


@pytest.mark.parametrize("n", [1, 2, 3])
def test_trace_tiny_trees(cuda, n):
    tris = scenes.gaussian_soup(n, clusters=1, seed=50 + n)
    b, t, out = G.build(tris)
    c = tris.reshape(-1, 3).mean(0)
    rays = scenes.random_rays(5000, c - 0.01, c + 0.01, seed=n)
    for q, m in ALL:
        np.testing.assert_array_equal(G.trace(b, t, rays, q, m),
                                      O.trace(out["nodes"], tris, out["root"], rays, q, m))


def test_trace_full_size_soup(cuda):
    tris = scenes.gaussian_soup()
    b, t, out = G.build(tris)
    rays = scenes.random_rays(100000, [0, 0, 0], [1, 1, 1], seed=9)
    rays[::2, 7] = 0.1
    for q in (0, 1):
        want = O.trace(out["nodes"], tris, out["root"], rays, q, 0)
        np.testing.assert_array_equal(G.trace(b, t, rays, q, 0), want)
        np.testing.assert_array_equal(G.trace(b, t, rays, q, 3), want)
