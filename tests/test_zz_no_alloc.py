"""mlbvh_build_noalloc: the build for callers that may not allocate device
memory (plugins whose host owns all GPU memory, real-time loops that cannot
take cudaMalloc's implicit synchronisation). It runs on a fixed device array
inside the library instead of caller scratch, so its results must equal
mlbvh_build's bit for bit, call after call, with nothing left over from the
previous call. This file sorts last so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import _gpu as G
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu


def noalloc_entry():
    f = mb.lib().mlbvh_build_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_build_equals_scratch_build(cuda):
    import torch
    build_noalloc = noalloc_entry()
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row; the second is smaller, so stale contents of the
    # first call's scratch would show in its output
    for n, seed in ((65536, 11), (4097, 12)):
        tris = scenes.gaussian_soup(n, clusters=8, seed=seed)
        t = G.dev(tris)
        ref = mb.BVHGPUBuilder().build(t, n, 0, mb.OnesweepSort())
        nodes = torch.empty((n - 1, 16), dtype=torch.int32, device="cuda")
        root = torch.empty(4, dtype=torch.int32, device="cuda")
        scene = torch.empty(8, dtype=torch.float32, device="cuda")
        status = build_noalloc(t.data_ptr(), n, 0, nodes.data_ptr(), root.data_ptr(), scene.data_ptr(), stream)
        assert status == 0, mb.lib().mlbvh_last_error_string()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(G.host(nodes), G.host(ref.m_internals)[: n - 1])
        assert int(G.host(root)[0]) == int(G.host(ref.m_rootNode)[0])
        np.testing.assert_array_equal(G.host(scene)[:6], G.host(ref.m_sceneAABB)[:6])


def test_noalloc_rejects_more_than_its_limit(cuda):
    build_noalloc = noalloc_entry()
    status = build_noalloc(256, 65537, 0, 256, 256, None, None)
    assert status == 1
    assert b"65536" in mb.lib().mlbvh_last_error_string()
