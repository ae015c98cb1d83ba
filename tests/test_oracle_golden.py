"""The oracle (oracle/mlbvh_oracle.c) against the reference's own known-answer
tests and the golden fixtures generated from the reference (tests/golden/).
CPU only."""
import os

import numpy as np
import pytest

import _oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_splat3_exhaustive_bits():
    """unittest.cpp:10-19: splat3 puts bit i of x at bit 3i; compact3 inverts it."""
    L = O.oracle()
    xs = np.arange(0, 1 << 21, 4093, dtype=np.uint32)
    for x in xs.tolist() + [0, 1, (1 << 21) - 1]:
        s = L.orc_splat3(x)
        for i in range(21):
            assert ((s >> (3 * i)) & 1) == ((x >> i) & 1)
        assert s & ~0x1249249249249249 == 0
        assert L.orc_compact3(s) == x


def test_morton_matches_naive_and_roundtrips():
    """unittest.cpp:21-36 with numpy's PCG64 in place of pr::PCG."""
    L = O.oracle()
    rng = np.random.default_rng(0)
    v = rng.integers(0, 1 << 21, (20000, 3), dtype=np.uint64)
    x = np.zeros(1, np.uint32)
    y = np.zeros(1, np.uint32)
    z = np.zeros(1, np.uint32)
    for a, b, c in v.tolist():
        m0 = L.orc_encode_morton_naive(a, b, c)
        assert m0 == L.orc_encode_morton(a, b, c)
        L.orc_decode_morton(m0, O.P(x), O.P(y), O.P(z))
        assert (int(x[0]), int(y[0]), int(z[0])) == (a, b, c)


def test_clz_ffs_known_answers():
    """unittest.cpp:39-105."""
    L = O.oracle()
    assert L.orc_clz(0) == 32 and L.orc_clz64(0) == 64
    assert L.orc_ffs(0) == 0 and L.orc_ffs64(0) == 0
    for i in range(32):
        v = 0x80000000 >> i
        assert L.orc_clz(v) == i and L.orc_clz(v | (v - 1)) == i
        u = 1 << i
        assert L.orc_ffs(u) == i + 1 and L.orc_ffs(u | (~(u - 1) & 0xFFFFFFFF)) == i + 1
    for i in range(64):
        v = 0x8000000000000000 >> i
        assert L.orc_clz64(v) == i and L.orc_clz64(v | (v - 1)) == i
        u = 1 << i
        assert L.orc_ffs64(u) == i + 1 and L.orc_ffs64(u | (~(u - 1) & 0xFFFFFFFFFFFFFFFF)) == i + 1


def test_morton_golden():
    L = O.oracle()
    g = load("morton_kat.npz")
    for v, c in zip(g["xyz"].tolist(), g["codes"].tolist()):
        assert L.orc_encode_morton(*v) == c
    for v, s in zip(g["splat_in"].tolist(), g["splat"].tolist()):
        assert L.orc_splat3(v) == s
    for v, c, f in zip(g["clz_in"].tolist(), g["clz_out"].tolist(), g["ffs_out"].tolist()):
        assert L.orc_clz(v) == c and L.orc_ffs(v) == f
    # AABB::encodeMortonCode incl. degenerate axes and points outside the box
    keys = np.zeros(1, np.uint32)
    for lo, hi, p, c in zip(g["box_lo"], g["box_hi"], g["box_p"], g["box_codes"].tolist()):
        box = np.concatenate([lo, hi]).astype(np.float32)
        tri = np.tile(p, 3).astype(np.float32)  # centroid of three equal points is p
        L.orc_morton_keys(O.P(tri), 1, 0, O.P(box), O.P(keys))
        assert int(keys[0]) == (c >> 31)


def test_toy_tree_golden():
    """main.cpp:60-109: the 8-key toy tree, built serially, validate_lbvh holds."""
    g = load("toy_tree.npz")
    keys = g["keys"]
    idx = np.arange(8, dtype=np.uint32)
    nodes = np.zeros((7, 16), np.uint32)
    deltas = np.zeros(7, np.uint8)
    root = np.zeros(1, np.uint32)
    # no triangles: bounds stay empty, as in the reference's toy run
    tris = np.zeros((8, 9), np.float32)
    L = O.oracle()
    L.orc_build_from_keys(O.P(keys), O.P(idx), O.P(tris), 8, O.P(nodes), O.P(deltas), O.P(root))
    np.testing.assert_array_equal(deltas, g["deltas"])
    assert int(root[0]) == int(g["root"][0])
    gn = g["nodes"]
    # topology, parent and context words (bounds differ: the toy run has no triangles)
    for col in (0, 1, 14, 15):
        np.testing.assert_array_equal(nodes[:, col], gn[:, col])
    assert L.orc_validate(O.P(nodes), O.P(deltas), 8, int(root[0]), 1 << 30) == 1


BUILD_CASES = ["soup1", "soup2", "soup3", "soup257", "soup4097", "dup300", "small_scene", "normal1000"]


@pytest.mark.parametrize("case", BUILD_CASES)
def test_build_golden(case):
    g = load("builds.npz")
    tris = g[f"{case}/tris"]
    b = O.build(tris, int(g[f"{case}/option"][0]))
    for k in ("keys", "indices", "deltas", "nodes"):
        np.testing.assert_array_equal(b[k], g[f"{case}/{k}"], err_msg=k)
    assert b["root"] == int(g[f"{case}/root"][0])
    np.testing.assert_array_equal(b["scene"], g[f"{case}/scene"])
    n = len(tris)
    if n > 1:
        L = O.oracle()
        assert L.orc_validate(O.P(b["nodes"]), O.P(b["deltas"]), n, b["root"], 255) == 1
        assert L.orc_check_tree(O.P(b["nodes"]), O.P(np.ascontiguousarray(tris)), n, b["root"]) == 1


@pytest.mark.parametrize("q,m", [(0, 0), (1, 0), (0, 1), (1, 1), (0, 2)])
def test_trace_golden(q, m):
    g = load("builds.npz")
    tris = g["small_scene/tris"]
    b = O.build(tris)
    t = load("traces.npz")
    np.testing.assert_array_equal(O.trace(b["nodes"], tris, b["root"], t["rays"], q, m), t[f"hits_q{q}_m{m}"])
    np.testing.assert_array_equal(O.trace(b["nodes"], tris, b["root"], t["short_rays"], q, m),
                                  t[f"short_q{q}_m{m}"])


def test_shading_golden():
    g = load("builds.npz")
    tris = g["small_scene/tris"]
    b = O.build(tris)
    s = load("shading.npz")
    w, h = s["size"].tolist()
    cam = s["camera"]
    # the reference's libm sin/cos (trig=0); PCG pairs in g++ argument order (mode 2)
    px, _ = O.render_ao(cam, b["root"], b["nodes"], tris, w, h, 16, 1.0, 12345, 1, trig=0)
    np.testing.assert_array_equal(px, s["ao_sobol"])
    px, _ = O.render_ao(cam, b["root"], b["nodes"], tris, w, h, 16, 1.0, 12345, 2, trig=0)
    np.testing.assert_array_equal(px, s["ao_pcg"])
    np.testing.assert_array_equal(O.render_normal(cam, b["root"], b["nodes"], tris, w, h), s["normal"])
    acc = np.zeros((w * h, 4), np.float32)
    for _ in range(2):
        O.render_pt(acc, cam, b["root"], b["nodes"], tris, s["attribs"], w, h, 1, trig=0)
    np.testing.assert_array_equal(acc, s["pt_sobol_2spp"])
    np.testing.assert_array_equal(O.pack(acc, w * h), s["pack"])
    acc = np.zeros((w * h, 4), np.float32)
    O.render_pt(acc, cam, b["root"], b["nodes"], tris, s["attribs"], w, h, 2, trig=0)
    np.testing.assert_array_equal(acc, s["pt_pcg_1spp"])


def test_samples_golden():
    L = O.oracle()
    g = load("samples.npz")
    xy = np.zeros(2, np.float32)
    x = np.zeros(1, np.float32)
    y = np.zeros(1, np.float32)
    for args, exp in zip(g["sobol_in"].tolist(), g["sobol_out"]):
        L.orc_sobol(*args, O.P(x), O.P(y))
        xy[:] = (x[0], y[0])
        np.testing.assert_array_equal(xy, exp)
    for v, e in zip(g["hash_in"].tolist(), g["hash_out"].tolist()):
        assert L.orc_hash_pcg(v) == e


def test_portable_sincos_accuracy():
    """The project's FP32 sincos (shared by oracle and kernels) stays within
    2 ulp of the true values over the hemisphere-sampling range [0, 2*pi)."""
    L = O.oracle()
    u = np.concatenate([np.linspace(0, 1, 20001, endpoint=False, dtype=np.float32),
                        np.random.default_rng(3).random(20000, dtype=np.float32)])
    phi = (u * np.float32(2.0)) * np.float32(np.pi)
    s = np.zeros(1, np.float32)
    c = np.zeros(1, np.float32)
    worst = 0.0
    for p in phi.tolist():
        L.orc_sincos(p, O.P(s), O.P(c))
        ts, tc = np.sin(np.float64(np.float32(p))), np.cos(np.float64(np.float32(p)))
        for got, true in ((s[0], ts), (c[0], tc)):
            ulp = np.spacing(np.float32(max(abs(true), 1e-30)))
            err = abs(float(got) - true)
            # near zeros of sin/cos measure against the ulp of the argument scale
            worst = max(worst, err / max(float(ulp), float(np.spacing(np.float32(1.0))) * 0.5))
    assert worst <= 2.0, worst
