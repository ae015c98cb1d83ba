"""mlbvh_build_noalloc: the build for callers that may not allocate device
memory (plugins whose host owns all GPU memory, real-time loops that cannot
take cudaMalloc's implicit synchronisation). It runs on a fixed device array
inside the library instead of caller scratch, so its results must equal
mlbvh_build's bit for bit, call after call, with nothing left over from the
previous call: across sizes (1 and 2 triangles included), with normal keys,
and on a second stream after a larger call on another. A timeout of its
bounded waits must be visible through mlbvh_scratch_status(NULL, stream).
This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
TIMEOUT = 3


def noalloc_entry():
    f = mb.lib().mlbvh_build_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def noalloc_status(stream):
    return mb.lib().mlbvh_scratch_status(None, stream)


def outputs(n, device="cuda"):
    import torch
    nodes = torch.empty((max(n - 1, 1), 16), dtype=torch.int32, device=device)
    root = torch.empty(4, dtype=torch.int32, device=device)
    scene = torch.empty(8, dtype=torch.float32, device=device)
    return nodes, root, scene


def check_equal(n, nodes, root, scene, ref):
    np.testing.assert_array_equal(G.host(nodes)[: n - 1], G.host(ref.m_internals)[: n - 1])
    assert int(G.host(root)[0]) == int(G.host(ref.m_rootNode)[0])
    np.testing.assert_array_equal(G.host(scene)[:6], G.host(ref.m_sceneAABB)[:6])


def scene_of(n, seed):
    if n <= 2:
        rng = np.random.default_rng(seed)
        return rng.uniform(-1, 1, (n, 9)).astype(np.float32)
    return scenes.gaussian_soup(n, clusters=8, seed=seed)


@pytest.mark.parametrize("option", [0, mb.BUILD_OPTION_USE_NORMAL])
def test_noalloc_build_equals_scratch_build(cuda, option):
    import torch
    build_noalloc = noalloc_entry()
    stream = torch.cuda.current_stream().cuda_stream
    # calls in a row; each is smaller than the one before, so stale contents
    # of an earlier call's scratch would show in the later outputs
    for n, seed in ((65536, 11), (4097, 12), (2, 13), (1, 14)):
        tris = scene_of(n, seed)
        t = G.dev(tris)
        ref = mb.BVHGPUBuilder().build(t, n, option, mb.OnesweepSort())
        nodes, root, scene = outputs(n)
        status = build_noalloc(t.data_ptr(), n, option, nodes.data_ptr() if n > 1 else None, root.data_ptr(),
                               scene.data_ptr(), stream)
        assert status == 0, mb.lib().mlbvh_last_error_string()
        assert noalloc_status(stream) == 0, mb.lib().mlbvh_last_error_string()
        torch.cuda.synchronize()
        check_equal(n, nodes, root, scene, ref)


def test_noalloc_second_stream_after_larger_call(cuda):
    """Calls serialised by the caller may run on different streams: a large
    call on one stream, synchronised, then a smaller one on another."""
    import torch
    build_noalloc = noalloc_entry()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    big = scenes.gaussian_soup(60000, clusters=8, seed=21)
    small = scenes.gaussian_soup(3000, clusters=4, seed=22)
    tb, ts = G.dev(big), G.dev(small)
    torch.cuda.synchronize()
    ob, os_ = outputs(len(big)), outputs(len(small))
    assert build_noalloc(tb.data_ptr(), len(big), 0, ob[0].data_ptr(), ob[1].data_ptr(), ob[2].data_ptr(),
                         s1.cuda_stream) == 0
    s1.synchronize()
    assert build_noalloc(ts.data_ptr(), len(small), 0, os_[0].data_ptr(), os_[1].data_ptr(), os_[2].data_ptr(),
                         s2.cuda_stream) == 0
    assert noalloc_status(s2.cuda_stream) == 0, mb.lib().mlbvh_last_error_string()
    torch.cuda.synchronize()
    check_equal(len(big), *ob, mb.BVHGPUBuilder().build(tb, len(big), 0, mb.OnesweepSort()))
    check_equal(len(small), *os_, mb.BVHGPUBuilder().build(ts, len(small), 0, mb.OnesweepSort()))


def test_noalloc_timeout_is_reported(cuda):
    """With the bounded waits cut to one poll (mlbvh_set_spin_limit), a call
    either reports MLBVH_ERR_TIMEOUT through mlbvh_scratch_status(NULL, ...)
    or built the oracle's tree; the next call with the default limit is the
    oracle's tree again."""
    import torch
    build_noalloc = noalloc_entry()
    stream = torch.cuda.current_stream().cuda_stream
    tris = scenes.gaussian_soup(65536, clusters=8, seed=41)
    n = len(tris)
    t = G.dev(tris)
    ref = O.build(tris)
    nodes, root, scene = outputs(n)

    def same_as_oracle():
        torch.cuda.synchronize()
        return bool((G.host(nodes, np.uint32)[: n - 1] == ref["nodes"]).all()) and \
            int(G.host(root, np.uint32)[0]) == ref["root"]

    L = mb.lib()
    timeouts = 0
    L.mlbvh_set_spin_limit(1)
    try:
        for _ in range(5):
            assert build_noalloc(t.data_ptr(), n, 0, nodes.data_ptr(), root.data_ptr(), scene.data_ptr(),
                                 stream) == 0
            s = noalloc_status(stream)
            if s == TIMEOUT:
                timeouts += 1
                continue
            assert s == 0, L.mlbvh_last_error_string()
            assert same_as_oracle(), "a call that reported no timeout must be the oracle's tree"
    finally:
        L.mlbvh_set_spin_limit(0)
    # one poll is far shorter than a sort tile's work: some wait gives up
    assert timeouts >= 1
    assert build_noalloc(t.data_ptr(), n, 0, nodes.data_ptr(), root.data_ptr(), scene.data_ptr(), stream) == 0
    assert noalloc_status(stream) == 0, L.mlbvh_last_error_string()
    assert same_as_oracle()


def test_noalloc_rejects_more_than_its_limit(cuda):
    build_noalloc = noalloc_entry()
    status = build_noalloc(256, 65537, 0, 256, 256, None, None)
    assert status == 1
    assert b"65536" in mb.lib().mlbvh_last_error_string()
