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


MISS = 0xFFFFFFFF


def _binary_boxes(nodes, n):
    """Box of every internal node (from its parent) and of every leaf
    position, as uint32 words."""
    box_int, box_leaf = {}, {}
    for j in range(n - 1):
        for s in (0, 1):
            c = int(nodes[j, s])
            box = nodes[j, 2 + 6 * s: 8 + 6 * s]
            if c & O.LEAF:
                box_leaf[j + s] = box
            else:
                box_int[c] = box
    return box_int, box_leaf


def test_wide_tree_regroups_the_binary_tree(case):
    """From the root, the wide slots reach every leaf position exactly once,
    each child with the binary tree's own box, two to four children a slot
    (non-empty slots first)."""
    _, tris, b, _, _ = case
    n = len(tris)
    wide = O.build_wide(b["nodes"], n)
    box_int, box_leaf = _binary_boxes(b["nodes"], n)
    seen = np.zeros(n, np.int64)
    todo, visited = [int(b["root"])], 0
    while todo:
        w = todo.pop()
        visited += 1
        kids = wide[w, 24:28]
        filled = kids != MISS
        assert filled.sum() >= 2 and (filled[:filled.sum()]).all()
        assert (wide[w, 28:] == 0).all()
        for k in np.nonzero(filled)[0]:
            c = int(kids[k])
            got = np.array([wide[w, k], wide[w, 8 + k], wide[w, 16 + k], wide[w, 4 + k], wide[w, 12 + k],
                            wide[w, 20 + k]], np.uint32)
            ref = box_leaf[c & ~O.LEAF] if c & O.LEAF else box_int[c]
            np.testing.assert_array_equal(got, ref)
            if c & O.LEAF:
                seen[c & ~O.LEAF] += 1
            else:
                todo.append(c)
    assert (seen == 1).all()
    assert visited < 0.6 * (n - 1)  # about half the binary nodes are slots the walk uses


def test_wide_any_hit_equals_stackfree(case):
    """Any-hit rays over the wide tree hit exactly when the stack-free walk's
    any-hit rays do, with fewer node visits; every reported hit is a real one."""
    name, tris, b, _, rays = case
    n = len(tris)
    wide = O.build_wide(b["nodes"], n)
    got, nv, nt, nr = O.trace_wide(wide, b["nodes"], tris, b["root"], rays)
    ref, nv0, _ = O.trace(b["nodes"], tris, b["root"], rays, 1, 0, counters=True)
    np.testing.assert_array_equal(got[:, 7] == MISS, ref[:, 7] == MISS)
    hit = got[:, 7] != MISS
    t = got[hit, 0].view(np.float32)
    assert (t >= rays[hit, 3]).all() and (t <= rays[hit, 7]).all()
    # the reported triangle, tested alone, gives the same t
    for i in np.nonzero(hit)[0][:50]:
        one = O.trace(np.zeros((0, 16), np.uint32), tris[got[i, 7]][None], O.LEAF, rays[i][None], 1, 0)
        assert one[0, 0] == got[i, 0]
    if name != "duplicates":
        assert nv.sum() < 0.7 * nv0.sum()
        assert nr.sum() == 0


def test_wide_stack_overflow_restarts_with_stackfree_walk():
    """Rays parallel to a triangle duplicated 400 times pass all its copies'
    boxes and miss them all: the wide stack overflows, the ray restarts with
    the stack-free walk, and hit/miss still equal the stack-free walk's."""
    base = scenes.gaussian_soup(3, seed=6)
    tris = np.tile(base, (400, 1))
    b = O.build(tris)
    wide = O.build_wide(b["nodes"], len(tris))
    v = base[0].reshape(3, 3).astype(np.float64)
    nrm = np.cross(v[1] - v[0], v[2] - v[1])
    nrm /= np.linalg.norm(nrm)
    c = v.mean(0)
    rng = np.random.default_rng(3)
    rays = np.zeros((64, 8), np.float32)
    for i in range(64):
        d = np.cross(nrm, rng.standard_normal(3))
        d /= np.linalg.norm(d)
        rays[i, 0:3] = c + nrm * 1e-5 - d * 0.01
        rays[i, 4:7] = d
        rays[i, 7] = 0.02
    got, nv, nt, nr = O.trace_wide(wide, b["nodes"], tris, b["root"], rays)
    ref = O.trace(b["nodes"], tris, b["root"], rays, 1, 0)
    np.testing.assert_array_equal(got[:, 7] == MISS, ref[:, 7] == MISS)
    assert nr.sum() > 0


def _decode_slot_planes(q):
    """Per slot, child and axis: (lower, upper) plane values base + v(code)
    in float64 (exact for these scenes; checked), and the children."""
    base = q[:, 0:3].view(np.float32).astype(np.float64)
    scale_bits = q[:, 3:6]
    planes = np.zeros((len(q), 4, 3, 2))
    for a in range(3):
        for side in range(2):
            codes = q[:, 6 + 2 * a + side]
            for k in range(4):
                code = (codes >> (8 * k)) & 255
                v = (scale_bits[:, a] | (code << 8)).astype(np.uint32).view(np.float32).astype(np.float64)
                s = base[:, a] + v
                assert ((s - base[:, a]) == v).all()  # the float64 sum is exact
                planes[:, k, a, side] = s
    return planes


def test_quantised_wide_slots_contain_fp32_slots(case):
    """Every decoded child box of every quantised slot contains the FP32
    slot's box; children are carried over unchanged."""
    _, tris, b, _, _ = case
    n = len(tris)
    wide = O.build_wide(b["nodes"], n)
    q, ok = O.quantise_wide(wide, n)
    assert ok
    np.testing.assert_array_equal(q[:, 12:16], wide[:, 24:28])
    planes = _decode_slot_planes(q)
    wf = wide.view(np.float32).astype(np.float64)
    for k in range(4):
        filled = wide[:, 24 + k] != MISS
        for a in range(3):
            lo, hi = wf[:, 8 * a + k], wf[:, 8 * a + 4 + k]
            assert (planes[filled, k, a, 0] <= lo[filled]).all()
            assert (planes[filled, k, a, 1] >= hi[filled]).all()
    # the codes use the 8 bits: the mean upper-minus-lower gap is far below the node
    # extent (a few codes per child plane, not the whole range)
    ext = planes[:, :, :, 1].max(1) - planes[:, :, :, 0].min(1)
    assert (ext > 0).mean() > 0.9


def test_quantised_wide_any_hit_equals_stackfree(case):
    name, tris, b, _, rays = case
    n = len(tris)
    wide = O.build_wide(b["nodes"], n)
    q, _ = O.quantise_wide(wide, n)
    got, nv, nt, nr = O.trace_wide_quantised(q, b["nodes"], tris, b["root"], rays)
    ref = O.trace(b["nodes"], tris, b["root"], rays, 1, 0)
    np.testing.assert_array_equal(got[:, 7] == MISS, ref[:, 7] == MISS)
    fp32, nv32, _, _ = O.trace_wide(wide, b["nodes"], tris, b["root"], rays)
    if name != "duplicates":
        # decoded boxes contain the exact ones: at least the FP32 walk's visits, not many more
        assert nv.sum() >= nv32.sum() and nv.sum() < 1.3 * nv32.sum()


def _closest_equal(got, ref, tris, name):
    """Closest hits: every Hit word equal, except that where duplicated
    triangles give bit-identical t the walk order picks which one reports
    (then t, uv and the normal are equal and the triangle is a copy)."""
    if name != "duplicates":
        np.testing.assert_array_equal(got, ref)
        return
    np.testing.assert_array_equal(got[:, [0, 2, 3, 4, 5, 6]], ref[:, [0, 2, 3, 4, 5, 6]])
    hit = got[:, 7] != MISS
    np.testing.assert_array_equal(tris[got[hit, 7]], tris[ref[hit, 7]])


def test_wide_closest_hit_equals_stackfree(case):
    """Closest-hit rays over the wide tree report intersect_stackfree's Hit
    records, with fewer node visits."""
    name, tris, b, _, rays = case
    wide = O.build_wide(b["nodes"], len(tris))
    got, nv, nt, nr = O.trace_wide(wide, b["nodes"], tris, b["root"], rays, query=0)
    ref, nv0, _ = O.trace(b["nodes"], tris, b["root"], rays, 0, 0, counters=True)
    _closest_equal(got, ref, tris, name)
    if name != "duplicates":
        assert nv.sum() < 0.7 * nv0.sum()


def test_quantised_wide_closest_hit_equals_stackfree(case):
    """The same over the quantised slots (a hit counts only where the
    triangle's exact box passes too): the FP32 walk's Hit records, at most a
    few more visits."""
    name, tris, b, _, rays = case
    n = len(tris)
    wide = O.build_wide(b["nodes"], n)
    q, _ = O.quantise_wide(wide, n)
    got, nv, nt, nr = O.trace_wide_quantised(q, b["nodes"], tris, b["root"], rays, query=0)
    ref = O.trace(b["nodes"], tris, b["root"], rays, 0, 0)
    _closest_equal(got, ref, tris, name)
    _, nv32, _, _ = O.trace_wide(wide, b["nodes"], tris, b["root"], rays, query=0)
    if name != "duplicates":
        assert nv.sum() >= nv32.sum() and nv.sum() < 1.3 * nv32.sum()


def nested_triangles():
    """400 scaled copies of one triangle about its centroid, growing with the
    index (one Morton key: a chain), and 64 rays parallel to their plane just
    above it from outside the smallest copies: every box passes, the nearest
    child of each slot is the internal one (the union of the larger copies),
    and no triangle is hit."""
    base = scenes.gaussian_soup(3, seed=6)
    v = base[0].reshape(3, 3).astype(np.float64)
    c = v.mean(0)
    nrm = np.cross(v[1] - v[0], v[2] - v[1])
    nrm /= np.linalg.norm(nrm)
    tris = np.array([(c + s * (v - c)).reshape(9) for s in np.linspace(0.2, 2.0, 400)], np.float32)
    rng = np.random.default_rng(3)
    rays = np.zeros((64, 8), np.float32)
    for i in range(64):
        d = np.cross(nrm, rng.standard_normal(3))
        d /= np.linalg.norm(d)
        rays[i, 0:3] = c + nrm * 1e-5 - d * 0.1
        rays[i, 4:7] = d
        rays[i, 7] = 0.3
    return tris, rays


def test_wide_closest_stack_overflow_restarts_with_stackfree_walk():
    """The closest-hit walk enters the nearest child and pushes the others:
    on nested_triangles() that overflows the wide stack, the walk restarts
    with the stack-free walk and still reports the stack-free walk's hits."""
    tris, rays = nested_triangles()
    b = O.build(tris)
    wide = O.build_wide(b["nodes"], len(tris))
    for q in (None, O.quantise_wide(wide, len(tris))[0]):
        if q is None:
            got, nv, nt, nr = O.trace_wide(wide, b["nodes"], tris, b["root"], rays, query=0)
        else:
            got, nv, nt, nr = O.trace_wide_quantised(q, b["nodes"], tris, b["root"], rays, query=0)
        ref = O.trace(b["nodes"], tris, b["root"], rays, 0, 0)
        np.testing.assert_array_equal(got, ref)
        assert nr.sum() > 0


def test_quantised_wide_rays_with_zero_direction_components_take_the_stackfree_walk():
    """A ray with a zero direction component (the reference clamps its
    inverse to +-FLT_MAX) could overflow the quantised slots' FMA form, which
    would lose its culling (an earlier form visited up to 22,040 slots per
    such ray). Such rays take the stack-free walk over the binary tree: the
    reference's Hit records and visit counts exactly. Rays that fit keep the
    quantised walk, with the FP32 walk's hits."""
    tris = scenes.gaussian_soup(50000, clusters=8, seed=5)
    b = O.build(tris)
    wide = O.build_wide(b["nodes"], len(tris))
    q, _ = O.quantise_wide(wide, len(tris))
    rng = np.random.default_rng(8)
    rays = np.zeros((3000, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.2, 1.2, (3000, 3))
    d = rng.standard_normal((3000, 3))
    d[:2000][np.arange(2000), rng.integers(0, 3, 2000)] = 0.0  # one zero component
    d[:700:7, :] *= [0.0, 1.0, 0.0]                          # some rays along an axis
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = np.float32(3.402823466e38)
    zero = (rays[:, 4:7] == 0).any(1)
    for query in (1, 0):
        got, nv, nt, nr = O.trace_wide_quantised(q, b["nodes"], tris, b["root"], rays, query=query)
        sf, nv0, nt0 = O.trace(b["nodes"], tris, b["root"], rays, query, 0, counters=True)
        np.testing.assert_array_equal(got[zero], sf[zero])
        np.testing.assert_array_equal(nv[zero], nv0[zero])
        np.testing.assert_array_equal(nt[zero], nt0[zero])
        ref, nv32, _, _ = O.trace_wide(wide, b["nodes"], tris, b["root"], rays, query=query)
        if query:
            np.testing.assert_array_equal(got[:, 7] == MISS, ref[:, 7] == MISS)
        else:
            np.testing.assert_array_equal(got, ref)
        assert nv[~zero].sum() < 1.3 * nv32[~zero].sum() and nr.sum() == 0


def test_quantised_wide_slots_refuse_coordinates_beyond_2_60():
    """Slots whose base would reach 2^60 (coordinates about 1e19) are not
    quantised: the walks' FMA form needs every plane below 2^61."""
    rng = np.random.default_rng(10)
    tris = (rng.random((300, 9)).astype(np.float32) + np.float32(8.0)) * np.float32(2e18)
    b = O.build(tris)
    wide = O.build_wide(b["nodes"], len(tris))
    _, ok = O.quantise_wide(wide, len(tris))
    assert not ok
    _, ok = O.quantise_wide(O.build_wide(O.build(tris / np.float32(1e3))["nodes"], len(tris)), len(tris))
    assert ok


def test_quantised_wide_fallback_for_huge_extents():
    """Coordinates spread over about 1e37 cannot be quantised (codes beyond
    8 bits at every scale up to 2^127): the slots are flagged and every ray
    takes the stack-free walk, with the same hits."""
    rng = np.random.default_rng(9)
    tris = (rng.random((200, 9)).astype(np.float32) - np.float32(0.5)) * np.float32(2e37)
    b = O.build(tris)
    wide = O.build_wide(b["nodes"], len(tris))
    _, ok = O.quantise_wide(wide, len(tris))
    assert not ok
    rays = scenes.random_rays(500, [-1e37, -1e37, -1e37], [1e37, 1e37, 1e37], seed=2)
    rays[:, 7] = np.float32(3e37)
    got, _, _, _ = O.trace_wide_quantised(np.zeros((len(tris) - 1, 16), np.uint32), b["nodes"], tris, b["root"],
                                          rays, fallback=True)
    ref = O.trace(b["nodes"], tris, b["root"], rays, 1, 0)
    np.testing.assert_array_equal(got, ref)


def _round_dir(x, up):
    """The float32 next to the exact rational x in the direction `up`
    (float32 overflow: +-inf or +-FLT_MAX, as directed rounding gives)."""
    from fractions import Fraction
    f = np.float32(float(x))  # nearest or adjacent
    if not np.isfinite(f):
        big = np.float32(3.4028234663852886e38)
        if x > 0:
            return np.float32(np.inf) if up else big
        return -big if up else np.float32(-np.inf)
    if Fraction(float(f)) < x and up:
        f = np.nextafter(f, np.float32(np.inf))
    elif Fraction(float(f)) > x and not up:
        f = np.nextafter(f, np.float32(-np.inf))
    while up and Fraction(float(np.nextafter(f, np.float32(-np.inf)))) >= x:
        f = np.nextafter(f, np.float32(-np.inf))
    while not up and Fraction(float(np.nextafter(f, np.float32(np.inf)))) <= x:
        f = np.nextafter(f, np.float32(np.inf))
    return np.float32(f)


def test_directed_fma_emulation_is_exact():
    """The oracle's a * b + c rounded down / up (the emulation of __fmaf_rd /
    __fmaf_ru in the quantised walks) equals the exact rational result
    rounded in that direction: random operands over many binades, products
    that cancel the addend, subnormal results and overflow."""
    from fractions import Fraction
    rng = np.random.default_rng(5)
    cases = []
    for _ in range(3000):
        a, b, c = (np.float32(rng.standard_normal() * 2.0 ** rng.integers(-60, 60)) for _ in range(3))
        cases.append((a, b, c))
        cases.append((a, b, np.float32(-np.float64(a) * np.float64(b))))  # cancellation
    cases += [(np.float32(1e-30), np.float32(1e-15), np.float32(0)), (np.float32(3e38), np.float32(10), np.float32(1)),
              (np.float32(-3e38), np.float32(10), np.float32(-1)), (np.float32(1.5), np.float32(2), np.float32(-3)),
              (np.float32(1e-40), np.float32(0.5), np.float32(1e-45))]
    for a, b, c in cases:
        exact = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
        for up in (0, 1):
            got = np.float32(O.oracle().orc_fma_dir(float(a), float(b), float(c), up))
            want = _round_dir(exact, up)
            assert got == want or (np.isinf(got) and np.isinf(want) and got == want), (a, b, c, up, got, want)


def test_entry_margin_without_abs_after_clip():
    """The packed slab tests move an entry down by 2^-22 of itself rather
    than of its magnitude (entry - 2^-22 entry rounded down, no |.| in a
    packed FMA). After the clip to lo = max(0, tmin) that is the scalar form
    max(entry - 2^-22 |entry| rounded down, lo) on every finite entry: equal
    where entry >= 0, both negative (so lo) where entry < 0, including
    subnormal entries, signed zeros and -FLT_MAX (whose scalar margin
    overflows to -inf)."""
    m = np.float32(2.384185791015625e-07)  # 2^-22
    rng = np.random.default_rng(11)
    ens = [np.float32(s * rng.random() * 2.0 ** rng.integers(-149, 127)) for s in (1, -1) for _ in range(2000)]
    ens += [np.float32(v) for v in (0.0, -0.0, 1e-45, -1e-45, 3e-45, -3e-45, 1.17549435e-38, -1.17549435e-38,
                                    3.4028235e38, -3.4028235e38, 1.0, -1.0)]
    los = [np.float32(0.0), np.float32(1e-45), np.float32(1e-3), np.float32(2.5)]
    fma = O.oracle().orc_fma_dir
    for en in ens:
        scalar = np.float32(fma(float(abs(en)), float(-m), float(en), 0))
        packed = np.float32(fma(float(en), float(-m), float(en), 0))
        for lo in los:
            assert max(scalar, lo) == max(packed, lo), (en, lo, scalar, packed)



def _axis_rays(n, lo, hi, seed):
    """Random rays, a third of them with one direction component exactly 0
    (the reference clamps its inverse to +-FLT_MAX, outside the FMA form's
    range): those take the decoded-box slab test."""
    rays = scenes.random_rays(n, lo, hi, seed=seed)
    rays[0::3, 4 + (np.arange(0, n, 3) % 3)] = 0.0
    return rays


@pytest.mark.parametrize("scale,status", [(1.0, 0), (1e20, 1), (1e37, 2)])
def test_quantised_status_paths_find_fp32_hits(scale, status):
    """The quantised binary tree's three node tests: the FMA form (status 0,
    rays within its range), the reference's slabs on the decoded boxes
    (status bit 0: coordinates near 1e20 give bases beyond 2^60; also every
    ray outside the FMA form's range) and every box passing (status bit 1: a
    scale exponent above 127 at about 1e37). Each returns the FP32 tree's
    closest hits; the replay walk returns the stack-free walk's Hit records."""
    rng = np.random.default_rng(31)
    tris = ((rng.random((3000, 9)) - 0.5) * scale).astype(np.float32)
    b = O.build(tris)
    q = O.quantise(b, tris)
    assert int(q["header"][3]) == status
    if status != 2:
        assert O.oracle().orc_check_quantised(O.P(b["nodes"]), len(tris), O.P(q["qnodes"]), O.P(q["header"])) == 1
    rays = _axis_rays(3000, [-0.5 * scale] * 3, [0.5 * scale] * 3, seed=32)
    got = O.trace_quantised(q, rays, 0)
    plain = O.trace(b["nodes"], tris, b["root"], rays, 0, 0)
    np.testing.assert_array_equal(got[:, 7], plain[:, 7])
    np.testing.assert_array_equal(got[:, 0], plain[:, 0])
    np.testing.assert_array_equal(O.trace_quantised(q, rays, 0, stack_depth=4), got)
