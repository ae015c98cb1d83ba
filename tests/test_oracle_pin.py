"""The oracle against the reference's own CPU code run live here
(oracle/_ref/libmlbvh_ref.so, built from the reference's sources by
oracle/Makefile). Skipped where that library was not built. CPU only."""
import numpy as np
import pytest

import _oracle as O
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libmlbvh_ref.so not built")


@pytest.fixture(scope="module")
def heightfield():
    tris = scenes.heightfield_icospheres()
    return tris, O.build(tris)


def test_build_heightfield_equals_reference(heightfield):
    tris, b = heightfield
    r = O.ref_build(tris, 0, parallel=1)
    for k in ("keys", "indices", "deltas", "nodes", "scene"):
        np.testing.assert_array_equal(b[k], r[k], err_msg=k)
    assert b["root"] == r["root"]


def test_unstable_reference_build_differs_only_by_tie_order():
    """BVHCPUBuilder itself (std::sort, parallel build_lbvh) gives the same
    deltas and topology shape when the keys are unique; with duplicate keys
    only the order of equal keys (hence leaf ids) may differ."""
    tris = scenes.gaussian_soup(20000, clusters=16, seed=4)
    b = O.build(tris)
    n = len(tris)
    nodes = np.zeros((n - 1, 16), np.uint32)
    deltas = np.zeros(n - 1, np.uint8)
    root = np.zeros(1, np.uint32)
    O.ref().ref_cpu_builder(O.P(tris), n, 2, O.P(nodes), O.P(deltas), O.P(root))
    np.testing.assert_array_equal(deltas, b["deltas"])
    assert int(root[0]) == b["root"]
    inner = (nodes[:, 0:2] & O.LEAF) == 0
    np.testing.assert_array_equal(nodes[:, 0:2][inner], b["nodes"][:, 0:2][inner])
    np.testing.assert_array_equal(nodes[:, 14:16], b["nodes"][:, 14:16])


@pytest.mark.parametrize("q,m", [(0, 0), (1, 0), (0, 1), (1, 1), (0, 2)])
def test_trace_heightfield_equals_reference(heightfield, q, m):
    tris, b = heightfield
    rays = scenes.random_rays(50000, [-1, -0.3, -1], [1, 0.7, 1], seed=31)
    rays[::3, 7] = 0.25
    np.testing.assert_array_equal(O.trace(b["nodes"], tris, b["root"], rays, q, m),
                                  O.ref_trace(b["nodes"], tris, b["root"], rays, q, m))


def test_ao_parameters_equal_reference(heightfield):
    """The restated AO with libm trig equals the reference's ao body at the
    heightfield workload's parameters (16 samples, radius 0.25)."""
    tris, b = heightfield
    w, h = 160, 120
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = O.lookat(eye, c, up, fovy, w, h)
    _, occ = O.render_ao(cam, b["root"], b["nodes"], tris, w, h, 16, 0.25, 12345, 1, trig=0)
    ref_occ = np.zeros(w * h, np.uint32)
    O.ref().ref_ao_param(O.P(ref_occ), w, h, O.P(cam), b["root"], O.P(b["nodes"]), O.P(tris), 16, 0.25, 12345, 0, h,
                         None)
    np.testing.assert_array_equal(occ, ref_occ)


def test_portable_trig_flip_rate(heightfield):
    """The one deliberate departure: sample directions from the project's FP32
    sincos instead of libm's. Occlusion counts may move where an AO ray grazes
    geometry; the rate is measured and bounded here (about 1e-4 of pixels)."""
    tris, b = heightfield
    w, h = 256, 256
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = O.lookat(eye, c, up, fovy, w, h)
    _, occ_libm = O.render_ao(cam, b["root"], b["nodes"], tris, w, h, 16, 0.25, 12345, 1, trig=0)
    _, occ_port = O.render_ao(cam, b["root"], b["nodes"], tris, w, h, 16, 0.25, 12345, 1, trig=1)
    hit = occ_libm != 0xFFFFFFFF
    diff = (occ_libm != occ_port) & hit
    assert diff.mean() < 2e-3, diff.mean()
    assert np.abs(occ_libm[hit].astype(np.int64) - occ_port[hit].astype(np.int64)).max(initial=0) <= 2
