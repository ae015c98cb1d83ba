"""Helpers for the GPU parity tests: move numpy arrays to the device and run
the product through its C ABI (minimumlbvh_b200's ctypes layer)."""
from __future__ import annotations

import numpy as np

import minimumlbvh_b200 as mb


def dev(a: np.ndarray, device="cuda"):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a.copy()).to(device)


def host(t, dtype=None) -> np.ndarray:
    a = t.detach().cpu().numpy()
    if dtype is not None:
        a = a.view(dtype)
    return a


def build(tris: np.ndarray, option: int = 0, sorter=None, stream=None):
    """GPU build; returns (builder, dict of host copies like _oracle.build)."""
    import torch
    t = dev(np.ascontiguousarray(tris, np.float32).reshape(-1, 9))
    b = mb.BVHGPUBuilder()
    b.build(t, len(tris), option, sorter, stream=stream, keep_keys=True)
    b.status(stream)
    n = len(tris)
    torch.cuda.synchronize()
    out = dict(nodes=host(b.m_internals, np.uint32)[: n - 1], deltas=host(b.m_deltas)[: max(n - 1, 0)],
               root=int(host(b.m_rootNode, np.uint32)[0]), keys=host(b.m_sortedKeys, np.uint32),
               indices=host(b.m_sortedIndices, np.uint32), scene=host(b.m_sceneAABB)[:6])
    if n > 1:
        # refuse to hand a structurally broken tree to any traversal test
        import _oracle as O
        assert O.oracle().orc_check_tree(O.P(out["nodes"]), O.P(np.ascontiguousarray(tris, np.float32)), n,
                                         out["root"]) == 1, "GPU build produced an invalid tree"
    return b, t, out


def assert_build_equal(gpu: dict, ref: dict):
    n = len(gpu["keys"])
    np.testing.assert_array_equal(gpu["keys"], ref["keys"], err_msg="sorted Morton keys")
    np.testing.assert_array_equal(gpu["indices"], ref["indices"], err_msg="sorted permutation")
    np.testing.assert_array_equal(gpu["deltas"], ref["deltas"][: max(n - 1, 0)], err_msg="deltas")
    assert gpu["root"] == ref["root"], "root"
    if n > 1:
        bad = np.nonzero((gpu["nodes"] != ref["nodes"]).any(1))[0]
        assert bad.size == 0, f"{bad.size} nodes differ, first {bad[:5]}: {gpu['nodes'][bad[:2]]} vs {ref['nodes'][bad[:2]]}"
    # the scene box as values (a zero bound may differ only in sign)
    assert (gpu["scene"] == ref["scene"]).all(), (gpu["scene"], ref["scene"])


def trace(builder, tris_t, rays: np.ndarray, query=0, mode=0):
    r = dev(np.ascontiguousarray(rays, np.float32))
    h = mb.intersect(builder, tris_t, r, query, mode)
    return host(h, np.uint32)
