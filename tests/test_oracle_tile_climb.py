"""The tile climb's interior rule, on the CPU, against the oracle's trees.

The GPU builds (single mesh and batched) let the two walkers of a node meet
through shared memory when the node's leaf range lies inside the CTA's tile of
consecutive sorted leaves, and decide this from the split deltas alone: node p
is interior when delta(p) <= max delta[t0 - 1 .. p - 1] and delta(p) <
max delta[p + 1 .. t1], deltas across a tree boundary (and outside the batch)
counting as infinite. In the batched build a tile may hold the end of one
mesh and the start of the next. This file restates that rule in numpy and
checks it, node by node, against the leaf ranges of the trees the oracle
builds (orc_build_from_keys, build_lbvh of minimum_lbvh.h:284-361) for meshes
laid end to end: a node is flagged exactly when its range lies in its tile,
and no position that is not a node (the last leaf of a mesh) is flagged."""
import numpy as np
import pytest

import _oracle as O

INF = 0xFFFFFFFF


def split_delta(a, b):
    x = np.bitwise_xor(a.astype(np.uint64), b.astype(np.uint64))
    out = np.zeros(len(x), np.int64)
    nz = x != 0
    out[nz] = np.floor(np.log2(x[nz].astype(np.float64))).astype(np.int64) + 1
    return out  # 32 - clz(a ^ b)


def batch_deltas(keys, offsets):
    """delta(g) between sorted leaves g and g + 1 of the whole batch, INF
    where they belong to different meshes and at the last leaf."""
    N = len(keys)
    d = np.full(N, INF, np.int64)
    if N > 1:
        d[:-1] = split_delta(keys[:-1], keys[1:])
    d[np.asarray(offsets[1:], np.int64) - 1] = INF
    return d


def interior_flags(d, T):
    """tile_climb_prepare restated: per tile [t0, t1], the exclusive prefix
    maximum from delta(t0 - 1) and the suffix maximum up to delta(t1)."""
    N = len(d)
    flags = np.zeros(N, bool)
    for t0 in range(0, N, T):
        t1 = min(t0 + T - 1, N - 1)
        left = INF if t0 == 0 else d[t0 - 1]
        w = d[t0 : t1 + 1]  # delta(t0 .. t1)
        pre = np.maximum.accumulate(np.concatenate(([left], w)))[:-1]  # max delta(t0 - 1 .. p - 1)
        suf = np.zeros(len(w), np.int64)  # max delta(p + 1 .. t1)
        if len(w) > 1:
            suf[:-1] = np.maximum.accumulate(w[::-1])[::-1][1:]
        p = np.arange(t0, t1 + 1)
        flags[t0 : t1 + 1] = (p < t1) & (w <= pre) & (w < suf)
    return flags


def leaf_ranges(nodes, root, n):
    """[L, U] of every internal node of an oracle tree whose leaf indices are
    sorted positions (triangle i at position i)."""
    L = np.zeros(max(n - 1, 0), np.int64)
    U = np.zeros(max(n - 1, 0), np.int64)
    if n < 2:
        return L, U
    order, stack = [], [root]
    while stack:
        v = stack.pop()
        order.append(v)
        for c in nodes[v, :2]:
            if not c & 0x80000000:
                stack.append(int(c))
    for v in reversed(order):
        lo, hi = [], []
        for c in nodes[v, :2]:
            c = int(c)
            if c & 0x80000000:
                lo.append(c & 0x7FFFFFFF)
                hi.append(c & 0x7FFFFFFF)
            else:
                lo.append(L[c])
                hi.append(U[c])
        L[v], U[v] = min(lo), max(hi)
    return L, U


def oracle_tree(keys):
    n = len(keys)
    idx = np.arange(n, dtype=np.uint32)
    tris = np.zeros((n, 9), np.float32)
    nodes = np.zeros((max(n - 1, 1), 16), np.uint32)
    deltas = np.zeros(max(n - 1, 1), np.uint8)
    root = np.zeros(1, np.uint32)
    O.oracle().orc_build_from_keys(O.P(np.ascontiguousarray(keys, np.uint32)), O.P(idx), O.P(tris), n, O.P(nodes),
                                   O.P(deltas), O.P(root))
    return nodes, int(root[0])


def batch_of(sizes, key_bits, seed):
    rng = np.random.default_rng(seed)
    keys = [np.sort(rng.integers(0, 1 << key_bits, s, dtype=np.uint64)).astype(np.uint32) for s in sizes]
    return keys, np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)


CASES = {
    "single_leaf_meshes": [1] * 130,
    "tile_edges": [63, 1, 64, 65, 2, 200, 1, 127, 128, 129],
    "one_mesh": [3000],
    "random": list(np.random.default_rng(5).integers(1, 300, 40)),
}


@pytest.mark.parametrize("tile", [32, 64, 128])
@pytest.mark.parametrize("key_bits", [6, 30])
@pytest.mark.parametrize("case", sorted(CASES))
def test_interior_rule_matches_oracle_ranges(case, key_bits, tile):
    sizes = [int(s) for s in CASES[case]]
    keys, off = batch_of(sizes, key_bits, seed=len(sizes) * 31 + key_bits)
    allKeys = np.concatenate(keys)
    N = len(allKeys)
    flags = interior_flags(batch_deltas(allKeys, off), tile)
    truth = np.zeros(N, bool)
    for m, k in enumerate(keys):
        n, start = len(k), int(off[m])
        assert not flags[start + n - 1], "the last leaf of a mesh is no node"
        if n < 2:
            continue
        nodes, root = oracle_tree(k)
        L, U = leaf_ranges(nodes, root, n)
        p = np.arange(n - 1)
        t0 = ((start + p) // tile) * tile
        t1 = np.minimum(t0 + tile - 1, N - 1)
        truth[start + p] = (start + L >= t0) & (start + U <= t1)
        # the nearest-blocker ranges the rule rests on, for every node
        assert (L <= p).all() and (U >= p + 1).all()
    np.testing.assert_array_equal(flags, truth)
    if case == "one_mesh" and key_bits == 30:
        assert truth.mean() > 0.6  # most nodes of a large tree of distinct keys meet inside their tile
