"""The C-ABI library without a GPU: it loads, exports every entry point that
include/mlbvh.h declares, rejects bad arguments before touching a device, and
its host-side camera set-up rounds as the reference's does. CPU only."""
import ctypes
import os
import re

import numpy as np
import pytest

import _oracle as O
import minimumlbvh_b200 as mb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"MLBVH_API\s+[\w\s\*]+?\b(mlbvh_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = mb.lib()
    names = declared_symbols()
    assert len(names) >= 13
    for name in names:
        assert hasattr(L, name), name
    assert L.mlbvh_version() == 1


def test_scratch_sizes_are_monotonic_and_aligned():
    L = mb.lib()
    prev = 0
    for n in (1, 2, 3, 4096, 4097, 1 << 20, 4194304):
        s = L.mlbvh_build_scratch_bytes(n)
        assert s % 256 == 0 and s >= prev and s >= 16 * n
        prev = s
    assert L.mlbvh_render_scratch_bytes(1920, 1080) >= 36 * 1920 * 1080
    assert L.mlbvh_render_scratch_bytes(0, 5) == 0


@pytest.mark.parametrize("n", [0, 1 << 30])
def test_build_rejects_bad_sizes(n):
    L = mb.lib()
    st = L.mlbvh_build(ctypes.c_void_p(256), n, 0, ctypes.c_void_p(256), ctypes.c_void_p(256), None,
                       ctypes.c_void_p(256), 1 << 40, None)
    assert st == 1
    assert b"nTriangles" in L.mlbvh_last_error_string()


def test_build_rejects_null_and_misaligned():
    L = mb.lib()
    assert L.mlbvh_build(None, 10, 0, ctypes.c_void_p(256), ctypes.c_void_p(256), None, ctypes.c_void_p(256),
                         1 << 40, None) == 1
    assert L.mlbvh_build(ctypes.c_void_p(260), 10, 0, ctypes.c_void_p(256), ctypes.c_void_p(256), None,
                         ctypes.c_void_p(256), 1 << 40, None) == 1
    assert b"aligned" in L.mlbvh_last_error_string()
    # scratch too small
    assert L.mlbvh_build(ctypes.c_void_p(256), 10, 0, ctypes.c_void_p(256), ctypes.c_void_p(256), None,
                         ctypes.c_void_p(256), 16, None) == 1
    assert b"scratch" in L.mlbvh_last_error_string()


def test_ploc_build_rejects_bad_arguments():
    L = mb.lib()
    v = ctypes.c_void_p
    for n in (1, 2, 1025, 1 << 20):
        assert L.mlbvh_build_ploc_scratch_bytes(n) >= L.mlbvh_build_scratch_bytes(n) + 128 * n
    for n, radius, word in ((0, 8, b"nTriangles"), (1 << 30, 8, b"nTriangles"), (10, 0, b"radius"),
                            (10, 33, b"radius")):
        assert L.mlbvh_build_ploc(v(256), n, 0, radius, v(256), v(256), None, v(256), 1 << 40, None) == 1
        assert word in L.mlbvh_last_error_string()
    assert L.mlbvh_build_ploc(None, 10, 0, 8, v(256), v(256), None, v(256), 1 << 40, None) == 1
    assert L.mlbvh_build_ploc(v(264), 10, 0, 8, v(256), v(256), None, v(256), 1 << 40, None) == 1
    assert b"aligned" in L.mlbvh_last_error_string()
    need = L.mlbvh_build_ploc_scratch_bytes(10)
    assert L.mlbvh_build_ploc(v(256), 10, 0, 8, v(256), v(256), None, v(256), need - 1, None) == 1
    assert b"scratch" in L.mlbvh_last_error_string()


def test_trace_and_render_reject_bad_arguments():
    L = mb.lib()
    p = ctypes.c_void_p(256)
    assert L.mlbvh_trace(p, p, p, p, p, 4, 7, 0, None) == 1  # bad query
    assert L.mlbvh_trace(p, p, p, p, p, 4, 0, 9, None) == 1  # bad traversal
    assert L.mlbvh_trace(p, p, p, p, p, 0, 0, 0, None) == 0  # nothing to do
    cam = (ctypes.c_float * 9)()
    assert L.mlbvh_render_ao(p, None, 0, 10, ctypes.addressof(cam), p, p, p, 1, 16, 1.0, 1, None, p, 1 << 30,
                             None) == 1
    assert L.mlbvh_render_ao(p, None, 8, 8, ctypes.addressof(cam), p, p, p, 1, 0, 1.0, 1, None, p, 1 << 30,
                             None) == 1
    assert L.mlbvh_render_ao(p, None, 8, 8, None, p, p, p, 1, 16, 1.0, 1, None, p, 1 << 30, None) == 1
    assert L.mlbvh_render_pt(p, 8, 8, ctypes.addressof(cam), p, p, p, p, 1, 4, -1, None) == 1
    assert L.mlbvh_render_pt_ex(p, 8, 8, ctypes.addressof(cam), p, p, p, p, 1, 4, 8, 7, None, None) == 1  # traversal
    assert b"traversal" in L.mlbvh_last_error_string()
    assert L.mlbvh_render_pt_ex(p, 8, 8, None, p, p, p, p, 1, 4, 8, 3, None, None) == 1  # null camera


def test_camera_lookat_matches_reference():
    for (eye, c, up, fovy, w, h) in [((0, 1.6, 1.6), (0, 0, 0), (0, 1, 0), 0.785398, 512, 512),
                                     ((0.5, 0.5, -1.2), (0.5, 0.5, 0.5), (0, 1, 0), 0.6981317, 1920, 1080),
                                     ((3, -2, 7), (0.1, 0.2, 0.3), (0, 0, 1), 1.2, 333, 97)]:
        g = mb.RayGenerator().lookat(eye, c, up, fovy, w, h).as_array()
        np.testing.assert_array_equal(g, O.lookat(eye, c, up, fovy, w, h))
        if O.ref_available():
            r = np.zeros(9, np.float32)
            O.ref().ref_lookat(O.P(np.array(eye, np.float32)), O.P(np.array(c, np.float32)),
                               O.P(np.array(up, np.float32)), float(np.float32(fovy)), w, h, O.P(r))
            np.testing.assert_array_equal(g, r)


def _fake_batch(**kw):
    d = mb._Batch()
    p = 256
    d.dTriangles = d.dMeshTriangleOffsets = d.dInternals = d.dRootNodes = d.dScratch = p
    d.dRays = d.dMeshRayOffsets = d.dHits = p
    d.nMeshes, d.nTriangles, d.nRays, d.scratchBytes = 4, 100, 10, 1 << 40
    for k, v in kw.items():
        setattr(d, k, v)
    return d


def test_batched_entry_points_reject_bad_arguments():
    L = mb.lib()
    by = ctypes.byref
    assert L.mlbvh_build_batched(None, None, None) == 1
    assert L.mlbvh_build_batched(by(_fake_batch(nMeshes=0)), None, None) == 1
    assert L.mlbvh_build_batched(by(_fake_batch(nTriangles=3)), None, None) == 1  # fewer triangles than meshes
    assert L.mlbvh_build_batched(by(_fake_batch(dTriangles=260)), None, None) == 1
    assert b"aligned" in L.mlbvh_last_error_string()
    assert L.mlbvh_build_batched(by(_fake_batch(scratchBytes=64)), None, None) == 1
    assert b"scratch" in L.mlbvh_last_error_string()
    p = mb.BatchParams.default()
    for field, bad in (("digitBits", 9), ("traceBlock", 96), ("queueChunk", 0), ("refillLanes", 33), ("walk", 2)):
        q = mb.BatchParams.default()
        setattr(q, field, bad)
        assert L.mlbvh_build_batched(by(_fake_batch()), by(q), None) == 1, field
        assert field in L.mlbvh_last_error_string().decode()
    assert L.mlbvh_trace_batched(by(_fake_batch(rayQuery=3)), by(p), None) == 1
    assert L.mlbvh_trace_batched(by(_fake_batch(nRays=1 << 31)), by(p), None) == 1
    assert L.mlbvh_trace_batched(by(_fake_batch(nRays=0)), by(p), None) == 0  # nothing to do
    g = ctypes.c_void_p()
    assert L.mlbvh_batch_graph_create(by(_fake_batch()), by(p), 0, by(g)) == 1
    assert L.mlbvh_batch_graph_create(by(_fake_batch()), by(p), 3, None) == 1
    assert L.mlbvh_batch_graph_launch(None, None) == 1
    L.mlbvh_batch_graph_destroy(None)


def test_batch_scratch_sizes():
    L = mb.lib()
    assert L.mlbvh_batch_scratch_bytes(0, 10) == 0
    assert L.mlbvh_batch_scratch_bytes(10, 9) == 0
    assert L.mlbvh_batch_scratch_bytes(1 << 21, 1 << 22) == 0
    prev = 0
    for nm, n in ((1, 1), (1, 4097), (16, 100000), (1024, 30_779_048)):
        s = L.mlbvh_batch_scratch_bytes(nm, n)
        assert s % 256 == 0 and s > prev and s >= 20 * n
        prev = s
    # the 1-mesh batch needs no less than the single-mesh build
    assert L.mlbvh_batch_scratch_bytes(1, 1 << 20) >= L.mlbvh_build_scratch_bytes(1 << 20)


def test_wide_entry_points_reject_bad_arguments():
    L = mb.lib()
    p, odd = ctypes.c_void_p(256), ctypes.c_void_p(256 + 64)
    assert L.mlbvh_build_wide(p, p, 0, p, None) == 1  # no triangles
    assert L.mlbvh_build_wide(p, p, 1, None, None) == 0  # one triangle: no slots, nothing to do
    assert L.mlbvh_build_wide(p, p, 10, odd, None) == 1  # wide nodes must be 128-byte aligned
    assert b"aligned" in L.mlbvh_last_error_string()
    assert L.mlbvh_trace_wide(p, p, p, p, p, p, p, 4, 2, None, None) == 1  # no such query
    assert b"rayQuery" in L.mlbvh_last_error_string()
    assert L.mlbvh_trace_wide(odd, p, p, p, p, p, p, 4, 1, None, None) == 1
    assert L.mlbvh_trace_wide(p, p, p, p, p, p, p, 0, 1, None, None) == 0  # nothing to do
    cam = (ctypes.c_float * 9)()
    assert L.mlbvh_render_ao_wide(p, None, 8, 8, ctypes.addressof(cam), p, p, p, odd, p, 1, 16, 1.0, 1, None, p,
                                  1 << 30, None) == 1
    assert L.mlbvh_render_ao_wide(p, None, 8, 8, ctypes.addressof(cam), p, p, p, p, None, 1, 16, 1.0, 1, None, p,
                                  1 << 30, None) == 1
    # quantised wide slots
    assert L.mlbvh_quantise_wide(p, 10, p, None, None) == 1  # no status word
    assert L.mlbvh_quantise_wide(p, 0, p, p, None) == 1      # no triangles
    assert L.mlbvh_trace_wide_quantised(p, p, p, p, p, p, p, p, 4, 2, None, None) == 1  # no such query
    assert L.mlbvh_trace_wide_quantised(p, None, p, p, p, p, p, p, 4, 1, None, None) == 1  # no status word
    assert L.mlbvh_trace_wide_quantised(ctypes.c_void_p(256 + 16), p, p, p, p, p, p, p, 4, 1, None, None) == 1
    assert L.mlbvh_render_ao_wide_quantised(p, None, 8, 8, ctypes.addressof(cam), p, p, p, p, None, p, 1, 16, 1.0, 1,
                                            None, p, 1 << 30, None) == 1
