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
