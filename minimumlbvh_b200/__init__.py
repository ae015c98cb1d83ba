"""minimumlbvh_b200 — MinimumLBVH's build, query and shading path on B200.

The work is done by libmlbvh_b200.so (hand-written sm_100a kernels behind the
C ABI of include/mlbvh.h). This module is the Python host side: it loads that
library with ctypes and mirrors the reference's host interface
(minimum_lbvh.h, tinyhiponesweep.h, camera.h, main_gpu.cu launches) over
torch CUDA tensors, which serve only as device memory and streams.

There is no CPU fallback: every compute call goes to the GPU library, and
``lib()`` raises if the library is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "lib", "library_path", "MlbvhError", "BUILD_OPTION_USE_NORMAL", "BUILD_OPTION_CPU_PARALLEL",
    "RAY_QUERY_CLOSEST", "RAY_QUERY_ANY", "TRAVERSAL_STACKFREE", "TRAVERSAL_ESCAPE_LINK",
    "TRAVERSAL_STACKFULL", "TRAVERSAL_REPLAY", "OnesweepSort", "BVHGPUBuilder", "RayGenerator", "intersect",
    "WideBVH", "intersect_wide", "render_ao_wide",
    "render_normal", "render_ao", "render_pt", "pack", "profile_events", "FLT_MAX", "INVALID_NODE",
    "QuantisedBVH", "intersect_quantised", "render_ao_quantised", "pt_diff_render", "pt_diff_adjoint",
    "BatchParams", "BatchedBVH", "leaf_triangles", "load_obj", "read_probe",
]

BUILD_OPTION_USE_NORMAL = 1   # minimum_lbvh.h:44
BUILD_OPTION_CPU_PARALLEL = 2  # minimum_lbvh.h:45 (accepted, ignored: the build runs on the GPU)
RAY_QUERY_CLOSEST = 0          # minimum_lbvh.h:977
RAY_QUERY_ANY = 1              # minimum_lbvh.h:978
TRAVERSAL_STACKFREE = 0
TRAVERSAL_ESCAPE_LINK = 1
TRAVERSAL_STACKFULL = 2
TRAVERSAL_REPLAY = 3  # intersect_stackfree's hits from a stack of pending far children (no revisits)
FLT_MAX = float(np.float32(3.402823466e38))
INVALID_NODE = 0x7FFFFFFF

_STATUS = {0: "MLBVH_OK", 1: "MLBVH_ERR_INVALID_ARG", 2: "MLBVH_ERR_OOM", 3: "MLBVH_ERR_TIMEOUT",
           4: "MLBVH_ERR_LAUNCH", 5: "MLBVH_ERR_CUDA"}

library_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmlbvh_b200.so")


class MlbvhError(RuntimeError):
    """A non-OK mlbvh_status; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None
_vp = ctypes.c_void_p


def lib() -> ctypes.CDLL:
    """The loaded libmlbvh_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError(f"{library_path} is missing: build it with `make -C minimumlbvh_b200` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(library_path)
        u32, i32, f32, sz = ctypes.c_uint32, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
        sig = {
            "mlbvh_version": (i32, []),
            "mlbvh_last_error_string": (ctypes.c_char_p, []),
            "mlbvh_build_scratch_bytes": (sz, [u32]),
            "mlbvh_build": (i32, [_vp, u32, u32, _vp, _vp, _vp, _vp, sz, _vp]),
            "mlbvh_build_ex": (i32, [_vp, u32, u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, sz, _vp]),
            "mlbvh_build_ploc_scratch_bytes": (sz, [u32]),
            "mlbvh_build_ploc": (i32, [_vp, u32, u32, i32, _vp, _vp, _vp, _vp, sz, _vp]),
            "mlbvh_set_spin_limit": (None, [u32]),
            "mlbvh_scratch_status": (i32, [_vp, _vp]),
            "mlbvh_trace": (i32, [_vp, _vp, _vp, _vp, _vp, u32, i32, i32, _vp]),
            "mlbvh_render_scratch_bytes": (sz, [i32, i32]),
            "mlbvh_render_normal": (i32, [_vp, i32, i32, _vp, _vp, _vp, _vp, _vp]),
            "mlbvh_render_ao": (i32, [_vp, _vp, i32, i32, _vp, _vp, _vp, _vp, i32, i32, f32, u32, _vp, _vp, sz,
                                      _vp]),
            "mlbvh_render_pt": (i32, [_vp, i32, i32, _vp, _vp, _vp, _vp, _vp, i32, i32, i32, _vp]),
            "mlbvh_render_pt_ex": (i32, [_vp, i32, i32, _vp, _vp, _vp, _vp, _vp, i32, i32, i32, i32, _vp, _vp]),
            "mlbvh_render_ao_ex": (i32, [_vp, _vp, i32, i32, _vp, _vp, _vp, _vp, i32, i32, f32, u32, i32, _vp, _vp,
                                         _vp, sz, _vp]),
            "mlbvh_leaf_triangles": (i32, [_vp, _vp, _vp, u32, _vp, _vp]),
            "mlbvh_build_wide": (i32, [_vp, _vp, u32, _vp, _vp]),
            "mlbvh_trace_wide": (i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, u32, i32, _vp, _vp]),
            "mlbvh_render_ao_wide": (i32, [_vp, _vp, i32, i32, _vp, _vp, _vp, _vp, _vp, _vp, i32, i32, f32, u32, _vp,
                                           _vp, sz, _vp]),
            "mlbvh_quantise_wide": (i32, [_vp, u32, _vp, _vp, _vp]),
            "mlbvh_trace_wide_quantised": (i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, u32, i32, _vp, _vp]),
            "mlbvh_render_ao_wide_quantised": (i32, [_vp, _vp, i32, i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, i32, i32,
                                                     f32, u32, _vp, _vp, sz, _vp]),
            "mlbvh_obj_load": (i32, [ctypes.c_char_p, _vp]),
            "mlbvh_obj_triangle_count": (u32, [_vp]),
            "mlbvh_obj_triangles": (_vp, [_vp]),
            "mlbvh_obj_attribs": (_vp, [_vp]),
            "mlbvh_obj_free": (None, [_vp]),
            "mlbvh_pack": (i32, [_vp, _vp, i32, _vp]),
            "mlbvh_profile_events": (None, [_vp, _vp]),
            "mlbvh_quantise": (i32, [_vp, _vp, _vp, u32, _vp, _vp, _vp, _vp, _vp]),
            "mlbvh_trace_quantised": (i32, [_vp, _vp, _vp, _vp, _vp, _vp, u32, i32, _vp]),
            "mlbvh_trace_quantised_ex": (i32, [_vp, _vp, _vp, _vp, _vp, _vp, u32, i32, i32, _vp, _vp]),
            "mlbvh_render_ao_quantised": (i32, [_vp, _vp, i32, i32, _vp, _vp, _vp, _vp, _vp, i32, i32, f32, u32,
                                                _vp, _vp, sz, _vp]),
            "mlbvh_camera_lookat": (i32, [_vp, _vp, _vp, _vp, f32, i32, i32]),
            "mlbvh_pt_diff_render": (i32, [_vp, i32, i32, i32, i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
            "mlbvh_pt_diff_adjoint": (i32, [_vp, _vp, i32, i32, i32, i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
            "mlbvh_batch_scratch_bytes": (sz, [u32, u32]),
            "mlbvh_batch_params_default": (None, [_vp]),
            "mlbvh_build_batched": (i32, [_vp, _vp, _vp]),
            "mlbvh_trace_batched": (i32, [_vp, _vp, _vp]),
            "mlbvh_batch_autotune": (i32, [_vp, _vp, _vp, _vp, _vp]),
            "mlbvh_batch_graph_create": (i32, [_vp, _vp, i32, _vp]),
            "mlbvh_batch_graph_launch": (i32, [_vp, _vp]),
            "mlbvh_batch_graph_destroy": (None, [_vp]),
            "mlbvh_read_probe": (i32, [_vp, sz, i32, u32, _vp, _vp, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != 0:
        raise MlbvhError(status, lib().mlbvh_last_error_string().decode())


def _ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def _stream(stream) -> int | None:
    import torch
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _require_cuda(t, name: str):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


class RayGenerator:
    """camera.h:3-32. ``lookat`` is computed by the C ABI on the host;
    ``as_bytes`` is the 36-byte struct the kernels take by value."""

    def __init__(self):
        self.m_origin = np.zeros(3, np.float32)
        self.m_right = np.array([1, 0, 0], np.float32)
        self.m_up = np.array([0, 1, 0], np.float32)

    def lookat(self, eye, center, up, fovy, imageWidth, imageHeight):
        out = (ctypes.c_float * 9)()
        e = (ctypes.c_float * 3)(*eye)
        c = (ctypes.c_float * 3)(*center)
        u = (ctypes.c_float * 3)(*up)
        _check(lib().mlbvh_camera_lookat(ctypes.addressof(out), ctypes.addressof(e), ctypes.addressof(c),
                                         ctypes.addressof(u), float(fovy), int(imageWidth), int(imageHeight)))
        a = np.frombuffer(bytes(out), dtype=np.float32)
        self.m_origin, self.m_right, self.m_up = a[0:3].copy(), a[3:6].copy(), a[6:9].copy()
        return self

    def as_array(self) -> np.ndarray:
        return np.concatenate([self.m_origin, self.m_right, self.m_up]).astype(np.float32)

    @classmethod
    def from_array(cls, a) -> "RayGenerator":
        g = cls()
        a = np.asarray(a, np.float32)
        g.m_origin, g.m_right, g.m_up = a[0:3].copy(), a[3:6].copy(), a[6:9].copy()
        return g

    def _cstruct(self):
        return (ctypes.c_float * 9)(*self.as_array().tolist())


class OnesweepSort:
    """tinyhiponesweep::OnesweepSort (tinyhiponesweep.h:572-748): owns the
    persistent scratch of the build (histograms, look-back words, key/value
    ping-pong buffers), grown on demand."""

    def __init__(self, device=None):
        import torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.scratch = None

    def reserve(self, nbytes: int):
        import torch
        if self.scratch is None or self.scratch.numel() < nbytes:
            self.scratch = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self.scratch


class BVHGPUBuilder:
    """BVHGPUBuilder (minimum_lbvh.h:726-885) over libmlbvh_b200.so.

    ``build`` leaves ``m_internals`` (int32 tensor, nTriangles-1 rows of the
    16-word InternalNode), ``m_rootNode`` (device int32 tensor of one
    NodeIndex; kernels dereference it, as in the reference) and
    ``m_sceneAABB`` (6 floats). Unlike the reference it neither allocates per
    call nor synchronises nor prints: the build is stream-ordered."""

    def __init__(self, kernelPath=None, includeDir=None):
        # The reference compiles minimum_lbvh.cu at run time from these paths;
        # here the kernels are compiled ahead of time, so they are ignored.
        self.m_internals = None
        self.m_rootNode = None
        self.m_sceneAABB = None
        self.m_nTriangles = 0
        self.m_sortedKeys = None
        self.m_sortedIndices = None
        self.m_deltas = None

    def build(self, triangles, nTriangles: int | None = None, buildOption: int = 0, sorter: OnesweepSort | None = None,
              stream=None, keep_keys: bool = False):
        import torch
        _require_cuda(triangles, "triangles")
        n = int(nTriangles if nTriangles is not None else triangles.numel() // 9)
        if n <= 0 or triangles.numel() < 9 * n:
            raise MlbvhError(1, "nTriangles must be positive and fit the triangle tensor")
        dev = triangles.device
        if sorter is None:
            sorter = OnesweepSort(dev.index)
        scratch = sorter.reserve(lib().mlbvh_build_scratch_bytes(n))
        if self.m_internals is None or self.m_internals.shape[0] != max(n - 1, 1) or self.m_internals.device != dev:
            self.m_internals = torch.empty((max(n - 1, 1), 16), dtype=torch.int32, device=dev)
        if self.m_rootNode is None or self.m_rootNode.device != dev:
            self.m_rootNode = torch.empty(4, dtype=torch.int32, device=dev)
            self.m_sceneAABB = torch.empty(8, dtype=torch.float32, device=dev)
        if keep_keys:
            self.m_sortedKeys = torch.empty(n, dtype=torch.int32, device=dev)
            self.m_sortedIndices = torch.empty(n, dtype=torch.int32, device=dev)
            self.m_deltas = torch.empty(max(n, 16), dtype=torch.uint8, device=dev)
            _check(lib().mlbvh_build_ex(_ptr(triangles), n, int(buildOption), _ptr(self.m_internals),
                                        _ptr(self.m_rootNode), _ptr(self.m_sceneAABB), _ptr(self.m_sortedKeys),
                                        _ptr(self.m_sortedIndices), _ptr(self.m_deltas), _ptr(scratch),
                                        scratch.numel(), _stream(stream)))
        else:
            _check(lib().mlbvh_build(_ptr(triangles), n, int(buildOption), _ptr(self.m_internals),
                                     _ptr(self.m_rootNode), _ptr(self.m_sceneAABB), _ptr(scratch), scratch.numel(),
                                     _stream(stream)))
        self.m_nTriangles = n
        self._sorter = sorter
        return self

    def buildByPLOC(self, triangles, nTriangles: int | None = None, buildOption: int = 0,
                    sorter: OnesweepSort | None = None, radius: int = 8, stream=None):
        """The higher-quality build (mlbvh_build_ploc), the GPU counterpart of
        BVHCPUBuilder::buildByEmbree (minimum_lbvh.h:594-656): the same
        members, the same node layout and numbering conventions as ``build``,
        a tree of smaller surface-area cost."""
        import torch
        _require_cuda(triangles, "triangles")
        n = int(nTriangles if nTriangles is not None else triangles.numel() // 9)
        if n <= 0 or triangles.numel() < 9 * n:
            raise MlbvhError(1, "nTriangles must be positive and fit the triangle tensor")
        dev = triangles.device
        if sorter is None:
            sorter = OnesweepSort(dev.index)
        scratch = sorter.reserve(lib().mlbvh_build_ploc_scratch_bytes(n))
        if self.m_internals is None or self.m_internals.shape[0] != max(n - 1, 1) or self.m_internals.device != dev:
            self.m_internals = torch.empty((max(n - 1, 1), 16), dtype=torch.int32, device=dev)
        if self.m_rootNode is None or self.m_rootNode.device != dev:
            self.m_rootNode = torch.empty(4, dtype=torch.int32, device=dev)
            self.m_sceneAABB = torch.empty(8, dtype=torch.float32, device=dev)
        _check(lib().mlbvh_build_ploc(_ptr(triangles), n, int(buildOption), int(radius), _ptr(self.m_internals),
                                      _ptr(self.m_rootNode), _ptr(self.m_sceneAABB), _ptr(scratch), scratch.numel(),
                                      _stream(stream)))
        self.m_nTriangles = n
        self._sorter = sorter
        return self

    def status(self, stream=None) -> None:
        """Synchronise and raise MlbvhError(MLBVH_ERR_TIMEOUT) if a bounded wait
        of the last build gave up."""
        _check(lib().mlbvh_scratch_status(_ptr(self._sorter.scratch), _stream(stream)))

    def empty(self) -> bool:
        return self.m_nTriangles == 0

    @property
    def nodes(self):
        return self.m_internals[: max(self.m_nTriangles - 1, 0)]


def intersect(builder_or_nodes, triangles, rays, rayQuery: int = RAY_QUERY_CLOSEST,
              traversal: int = TRAVERSAL_STACKFREE, hits=None, root=None, stream=None):
    """One launch of intersect_stackfree / _escape_link / _stackfull
    (minimum_lbvh.h:981, 1063, 912) over ``rays`` (float32 (n, 8):
    ro.xyz, tmin, rd.xyz, tmax). Returns ``hits`` (int32 (n, 8) holding the
    32-byte Hit records)."""
    import torch
    if isinstance(builder_or_nodes, BVHGPUBuilder):
        nodes, root = builder_or_nodes.m_internals, builder_or_nodes.m_rootNode
    else:
        nodes = builder_or_nodes
    _require_cuda(rays, "rays")
    n = rays.numel() // 8
    if hits is None:
        hits = torch.empty((n, 8), dtype=torch.int32, device=rays.device)
    _check(lib().mlbvh_trace(_ptr(nodes), _ptr(root), _ptr(triangles), _ptr(rays), _ptr(hits), n, int(rayQuery),
                             int(traversal), _stream(stream)))
    return hits


def render_normal(pixels, imageSize, rayGenerator: RayGenerator, rootNode, internals, triangles, stream=None):
    """normal (main_gpu.cu:84-109)."""
    w, h = imageSize
    cam = rayGenerator._cstruct()
    _check(lib().mlbvh_render_normal(_ptr(pixels), int(w), int(h), ctypes.addressof(cam), _ptr(rootNode),
                                     _ptr(internals), _ptr(triangles), _stream(stream)))
    return pixels


_render_scratch = {}


def read_probe(buffer, pattern: int, loads: int, sink, stream=None) -> int:
    """mlbvh_read_probe: one launch reading ``buffer`` (a 32-byte aligned
    device tensor) with the traversal's 32-byte node load, streaming
    (pattern 0, ``loads`` sweeps) or gathering random sectors (pattern 1,
    ``loads`` per thread); ``sink`` is a device tensor of at least 1024 int32.
    Returns the bytes the launch reads; time it with CUDA events."""
    _require_cuda(buffer, "buffer")
    out = ctypes.c_size_t(0)
    _check(lib().mlbvh_read_probe(_ptr(buffer), buffer.numel() * buffer.element_size(), int(pattern), int(loads),
                                  _ptr(sink), ctypes.byref(out), _stream(stream)))
    return int(out.value)


def profile_events(start=None, stop=None):
    """Make the next render_ao / BVHGPUBuilder.build on this thread record
    the torch.cuda.Event pair around its dominant kernel."""
    for e in (start, stop):
        if e is not None and not e.cuda_event:
            e.record()  # torch creates the CUDA event on first record; the hook re-records it
    lib().mlbvh_profile_events(None if start is None else start.cuda_event,
                               None if stop is None else stop.cuda_event)


def _ao_scratch(pixels, w: int, h: int, scratch=None):
    """The caller's AO scratch, or a cached device buffer of the needed size."""
    import torch
    if scratch is not None:
        return scratch
    need = lib().mlbvh_render_scratch_bytes(int(w), int(h))
    key = (pixels.device.index, need)
    scratch = _render_scratch.get(key)
    if scratch is None:
        scratch = torch.empty(need, dtype=torch.uint8, device=pixels.device)
        _render_scratch.clear()
        _render_scratch[key] = scratch
    return scratch


def render_ao(pixels, imageSize, rayGenerator: RayGenerator, rootNode, internals, triangles, useSobol: int = 1,
              nSamples: int = 16, radius: float = 1.0, seed: int = 12345, occluded=None, stats=None,
              scratch=None, stream=None, traversal: int = TRAVERSAL_STACKFREE, leaf_triangles=None):
    """ao (main_gpu.cu:111-177) with sample count, radius and Sobol seed as
    parameters (the reference fixes 16, 1.0, 12345). ``stats`` (int64 CUDA
    tensor of 8) receives rays traced, node visits and triangle tests.
    ``traversal`` TRAVERSAL_REPLAY gives the same result from the replay walk,
    reading ``leaf_triangles`` (from ``leaf_triangles()``) when given."""
    w, h = imageSize
    scratch = _ao_scratch(pixels, w, h, scratch)
    cam = rayGenerator._cstruct()
    if traversal == TRAVERSAL_STACKFREE:
        _check(lib().mlbvh_render_ao(_ptr(pixels), _ptr(occluded), int(w), int(h), ctypes.addressof(cam),
                                     _ptr(rootNode), _ptr(internals), _ptr(triangles), int(useSobol), int(nSamples),
                                     float(radius), int(seed), _ptr(stats), _ptr(scratch), scratch.numel(),
                                     _stream(stream)))
    else:
        _check(lib().mlbvh_render_ao_ex(_ptr(pixels), _ptr(occluded), int(w), int(h), ctypes.addressof(cam),
                                        _ptr(rootNode), _ptr(internals), _ptr(triangles), int(useSobol),
                                        int(nSamples), float(radius), int(seed), int(traversal),
                                        _ptr(leaf_triangles), _ptr(stats), _ptr(scratch), scratch.numel(),
                                        _stream(stream)))
    return pixels


def leaf_triangles(builder: "BVHGPUBuilder", triangles, out=None, stream=None):
    """The built tree's triangles in leaf order as 48-byte records (int32
    (n, 12): corners, original index, padding), mlbvh_leaf_triangles."""
    import torch
    n = builder.m_nTriangles
    if out is None:
        out = torch.empty((n, 12), dtype=torch.int32, device=triangles.device)
    _check(lib().mlbvh_leaf_triangles(_ptr(builder.m_internals), _ptr(builder.m_rootNode), _ptr(triangles), n,
                                      _ptr(out), _stream(stream)))
    return out


class WideBVH:
    """The 4-wide tree of a built tree (mlbvh_build_wide) with the triangles
    in leaf order (mlbvh_leaf_triangles): any-hit rays over it find a hit
    exactly when the stack-free any-hit walk does, loading half as many
    nodes in a chain. Holds the builder's arrays for primary rays and for the
    restart of a ray whose stack would overflow."""

    def __init__(self, builder: "BVHGPUBuilder", triangles, wide, leaf_tris):
        self.builder, self.triangles, self.wide, self.leaf_triangles = builder, triangles, wide, leaf_tris
        self.qwide = None   # quantised slots (quantise())
        self.status = None  # int32 device word: 1 when a slot could not be quantised

    def quantise(self, stream=None) -> "WideBVH":
        """The 64-byte quantised slots (mlbvh_quantise_wide), kept beside the
        FP32 ones."""
        import torch
        n = self.builder.m_nTriangles
        if self.qwide is None:
            self.qwide = torch.empty((max(n - 1, 1), 16), dtype=torch.int32, device=self.wide.device)
            self.status = torch.zeros(4, dtype=torch.int32, device=self.wide.device)
        _check(lib().mlbvh_quantise_wide(_ptr(self.wide), n, _ptr(self.qwide), _ptr(self.status), _stream(stream)))
        return self

    @classmethod
    def from_builder(cls, builder: "BVHGPUBuilder", triangles, stream=None) -> "WideBVH":
        import torch
        n = builder.m_nTriangles
        wide = torch.empty((max(n - 1, 1), 32), dtype=torch.int32, device=triangles.device)
        _check(lib().mlbvh_build_wide(_ptr(builder.m_internals), _ptr(builder.m_rootNode), n, _ptr(wide),
                                      _stream(stream)))
        return cls(builder, triangles, wide, leaf_triangles(builder, triangles, stream=stream))

    def update(self, stream=None) -> "WideBVH":
        """Regroup again after the builder rebuilt its tree (same triangle
        count): the wide slots and the leaf-ordered triangles, in place."""
        n = self.builder.m_nTriangles
        _check(lib().mlbvh_build_wide(_ptr(self.builder.m_internals), _ptr(self.builder.m_rootNode), n,
                                      _ptr(self.wide), _stream(stream)))
        leaf_triangles(self.builder, self.triangles, out=self.leaf_triangles, stream=stream)
        if self.qwide is not None:
            self.quantise(stream)
        return self


def intersect_wide(w: WideBVH, rays, hits=None, counts=None, stream=None, quantised: bool = False,
                   rayQuery: int = RAY_QUERY_ANY):
    """Rays over the 4-wide tree (mlbvh_trace_wide, or with ``quantised``
    mlbvh_trace_wide_quantised over ``w.quantise()``'s slots), any-hit
    (default) or closest-hit (``rayQuery=RAY_QUERY_CLOSEST``: the stack-free
    walk's Hit records). ``counts`` (int32 CUDA tensor of 3 * nRays) receives
    per-ray node visits, triangle tests and restarts."""
    import torch
    _require_cuda(rays, "rays")
    n = rays.numel() // 8
    if hits is None:
        hits = torch.empty((n, 8), dtype=torch.int32, device=rays.device)
    b = w.builder
    if quantised:
        _check(lib().mlbvh_trace_wide_quantised(_ptr(w.qwide), _ptr(w.status), _ptr(b.m_internals),
                                                _ptr(b.m_rootNode), _ptr(w.triangles), _ptr(w.leaf_triangles),
                                                _ptr(rays), _ptr(hits), n, int(rayQuery), _ptr(counts),
                                                _stream(stream)))
    else:
        _check(lib().mlbvh_trace_wide(_ptr(w.wide), _ptr(b.m_internals), _ptr(b.m_rootNode), _ptr(w.triangles),
                                      _ptr(w.leaf_triangles), _ptr(rays), _ptr(hits), n, int(rayQuery),
                                      _ptr(counts), _stream(stream)))
    return hits


def render_ao_wide(pixels, imageSize, rayGenerator: RayGenerator, w: WideBVH, useSobol: int = 1,
                   nSamples: int = 16, radius: float = 1.0, seed: int = 12345, occluded=None, stats=None,
                   scratch=None, stream=None, quantised: bool = False):
    """render_ao with the AO rays over the 4-wide tree (same occlusion
    counts; ``quantised``: over ``w.quantise()``'s 64-byte slots) and primary
    rays on the replay walk (the same Hit records)."""
    width, height = imageSize
    scratch = _ao_scratch(pixels, width, height, scratch)
    cam = rayGenerator._cstruct()
    b = w.builder
    if quantised:
        _check(lib().mlbvh_render_ao_wide_quantised(
            _ptr(pixels), _ptr(occluded), int(width), int(height), ctypes.addressof(cam), _ptr(b.m_rootNode),
            _ptr(b.m_internals), _ptr(w.triangles), _ptr(w.qwide), _ptr(w.status), _ptr(w.leaf_triangles),
            int(useSobol), int(nSamples), float(radius), int(seed), _ptr(stats), _ptr(scratch), scratch.numel(),
            _stream(stream)))
    else:
        _check(lib().mlbvh_render_ao_wide(_ptr(pixels), _ptr(occluded), int(width), int(height),
                                          ctypes.addressof(cam), _ptr(b.m_rootNode), _ptr(b.m_internals),
                                          _ptr(w.triangles), _ptr(w.wide), _ptr(w.leaf_triangles), int(useSobol),
                                          int(nSamples), float(radius), int(seed), _ptr(stats), _ptr(scratch),
                                          scratch.numel(), _stream(stream)))
    return pixels


def render_pt(accumulators, imageSize, rayGenerator: RayGenerator, rootNode, internals, triangles,
              triangleAttribs, useSobol: int = 1, maxSPP: int = 1 << 30, maxDepth: int = 1024, stream=None,
              traversal: int = TRAVERSAL_STACKFREE, leaf_triangles=None):
    """One progressive pass of pt (main_gpu.cu:179-272). ``traversal``
    TRAVERSAL_REPLAY gives the same accumulators from the replay walk,
    reading ``leaf_triangles`` (from ``leaf_triangles()``) when given."""
    w, h = imageSize
    cam = rayGenerator._cstruct()
    if traversal == TRAVERSAL_STACKFREE and leaf_triangles is None:
        _check(lib().mlbvh_render_pt(_ptr(accumulators), int(w), int(h), ctypes.addressof(cam), _ptr(rootNode),
                                     _ptr(internals), _ptr(triangles), _ptr(triangleAttribs), int(useSobol),
                                     int(maxSPP), int(maxDepth), _stream(stream)))
    else:
        _check(lib().mlbvh_render_pt_ex(_ptr(accumulators), int(w), int(h), ctypes.addressof(cam), _ptr(rootNode),
                                        _ptr(internals), _ptr(triangles), _ptr(triangleAttribs), int(useSobol),
                                        int(maxSPP), int(maxDepth), int(traversal), _ptr(leaf_triangles),
                                        _stream(stream)))
    return accumulators


def pack(pixels, accumulators, n: int, stream=None):
    """pack (main_gpu.cu:273-286)."""
    _check(lib().mlbvh_pack(_ptr(pixels), _ptr(accumulators), int(n), _stream(stream)))
    return pixels


class QuantisedBVH:
    """The quantised form of a built tree (no reference counterpart):
    32-byte nodes with 8-bit child boxes rounded outward, a parent array and
    leaf-ordered triangles. ``from_builder`` converts a BVHGPUBuilder's tree
    on the GPU (mlbvh_quantise)."""

    def __init__(self, qnodes, parents, qtris, header, n):
        self.qnodes, self.parents, self.qtris, self.header, self.nTriangles = qnodes, parents, qtris, header, n

    @classmethod
    def from_builder(cls, builder: BVHGPUBuilder, triangles, stream=None) -> "QuantisedBVH":
        import torch
        n = builder.m_nTriangles
        dev = triangles.device
        qnodes = torch.empty((max(n - 1, 1), 8), dtype=torch.int32, device=dev)
        parents = torch.empty(max(n - 1, 1) + 3, dtype=torch.int32, device=dev)
        qtris = torch.empty((n, 12), dtype=torch.int32, device=dev)
        header = torch.empty(4, dtype=torch.int32, device=dev)
        _check(lib().mlbvh_quantise(_ptr(builder.m_internals), _ptr(builder.m_rootNode), _ptr(triangles), n,
                                    _ptr(qnodes), _ptr(parents), _ptr(qtris), _ptr(header), _stream(stream)))
        return cls(qnodes, parents, qtris, header, n)


def intersect_quantised(q: QuantisedBVH, rays, rayQuery: int = RAY_QUERY_CLOSEST, hits=None, stream=None,
                        stack_depth: int | None = None, counts=None):
    """Closest/any hit over the quantised tree (the stack-free walk's Hit
    records). ``stack_depth`` None: the library's default walk; 0: the
    stack-free walk; 1, 4 or 16: the replay walk with that many stack
    entries. ``counts`` (int32 CUDA tensor of 3 * nRays) receives per-ray
    node visits, triangle tests and parent loads."""
    import torch
    _require_cuda(rays, "rays")
    n = rays.numel() // 8
    if hits is None:
        hits = torch.empty((n, 8), dtype=torch.int32, device=rays.device)
    if stack_depth is None and counts is None:
        _check(lib().mlbvh_trace_quantised(_ptr(q.qnodes), _ptr(q.parents), _ptr(q.qtris), _ptr(q.header),
                                           _ptr(rays), _ptr(hits), n, int(rayQuery), _stream(stream)))
    else:
        _check(lib().mlbvh_trace_quantised_ex(_ptr(q.qnodes), _ptr(q.parents), _ptr(q.qtris), _ptr(q.header),
                                              _ptr(rays), _ptr(hits), n, int(rayQuery),
                                              16 if stack_depth is None else int(stack_depth), _ptr(counts),
                                              _stream(stream)))
    return hits


def render_ao_quantised(pixels, imageSize, rayGenerator: RayGenerator, q: QuantisedBVH, useSobol: int = 1,
                        nSamples: int = 16, radius: float = 1.0, seed: int = 12345, occluded=None, stats=None,
                        scratch=None, stream=None):
    """render_ao over the quantised tree."""
    w, h = imageSize
    scratch = _ao_scratch(pixels, w, h, scratch)
    cam = rayGenerator._cstruct()
    _check(lib().mlbvh_render_ao_quantised(_ptr(pixels), _ptr(occluded), int(w), int(h), ctypes.addressof(cam),
                                           _ptr(q.qnodes), _ptr(q.parents), _ptr(q.qtris), _ptr(q.header),
                                           int(useSobol), int(nSamples), float(radius), int(seed), _ptr(stats),
                                           _ptr(scratch), scratch.numel(), _stream(stream)))
    return pixels


def pt_diff_render(image, imageSize, rayGenerator: RayGenerator, builder: BVHGPUBuilder, triangles, albedo, emission,
                   spp: int, bounces: int = 3, stream=None):
    """Fixed-depth differentiable path trace (float image, one value per
    pixel) with per-triangle grey albedo and emission."""
    w, h = imageSize
    cam = rayGenerator._cstruct()
    _check(lib().mlbvh_pt_diff_render(_ptr(image), int(w), int(h), int(spp), int(bounces), ctypes.addressof(cam),
                                      _ptr(builder.m_rootNode), _ptr(builder.m_internals), _ptr(triangles),
                                      _ptr(albedo), _ptr(emission), _stream(stream)))
    return image


def pt_diff_adjoint(grad_albedo, grad_image, imageSize, rayGenerator: RayGenerator, builder: BVHGPUBuilder, triangles,
                    albedo, emission, spp: int, bounces: int = 3, stream=None):
    """Path-replay adjoint: ADDS dLoss/dAlbedo to grad_albedo given
    dLoss/dImage."""
    w, h = imageSize
    cam = rayGenerator._cstruct()
    _check(lib().mlbvh_pt_diff_adjoint(_ptr(grad_albedo), _ptr(grad_image), int(w), int(h), int(spp), int(bounces),
                                       ctypes.addressof(cam), _ptr(builder.m_rootNode), _ptr(builder.m_internals),
                                       _ptr(triangles), _ptr(albedo), _ptr(emission), _stream(stream)))
    return grad_albedo


class BatchParams(ctypes.Structure):
    """mlbvh_batch_params: launch parameters of the batched form."""
    _fields_ = [("digitBits", ctypes.c_int), ("traceBlock", ctypes.c_int), ("queueChunk", ctypes.c_int),
                ("refillLanes", ctypes.c_int), ("walk", ctypes.c_int)]

    @classmethod
    def default(cls) -> "BatchParams":
        p = cls()
        lib().mlbvh_batch_params_default(ctypes.byref(p))
        return p

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class _Batch(ctypes.Structure):
    _fields_ = [("dTriangles", _vp), ("dMeshTriangleOffsets", _vp), ("nMeshes", ctypes.c_uint32),
                ("nTriangles", ctypes.c_uint32), ("buildOption", ctypes.c_uint32), ("rayQuery", ctypes.c_int),
                ("dInternals", _vp), ("dRootNodes", _vp), ("dMeshAABBs", _vp), ("dRays", _vp),
                ("dMeshRayOffsets", _vp), ("nRays", ctypes.c_uint32), ("_pad", ctypes.c_uint32), ("dHits", _vp),
                ("dScratch", _vp), ("scratchBytes", ctypes.c_size_t)]


class BatchedBVH:
    """Many meshes built in one launch chain and traced by one persistent
    kernel (mlbvh_build_batched / mlbvh_trace_batched; no reference
    counterpart). ``triangles`` is float32 (nTriangles, 9) with the meshes back
    to back; ``tri_offsets`` (nMeshes + 1, int32 on the device) bounds them.
    After ``build``, ``internals`` (nTriangles - nMeshes rows of 16 words),
    ``roots`` (nMeshes) and ``mesh_aabbs`` (nMeshes x 6) hold the trees: mesh
    m's nodes start at row tri_offsets[m] - m."""

    def __init__(self, triangles, tri_offsets, n_meshes: int, buildOption: int = 0):
        import torch
        _require_cuda(triangles, "triangles")
        _require_cuda(tri_offsets, "tri_offsets")
        dev = triangles.device
        self.triangles, self.tri_offsets = triangles, tri_offsets
        self.nMeshes, self.nTriangles = int(n_meshes), triangles.numel() // 9
        nbytes = lib().mlbvh_batch_scratch_bytes(self.nMeshes, self.nTriangles)
        if nbytes == 0:
            raise MlbvhError(1, "nMeshes must be in [1, 2^20] and nTriangles in [nMeshes, 2^30)")
        self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.internals = torch.empty((max(self.nTriangles - self.nMeshes, 1), 16), dtype=torch.int32, device=dev)
        self.roots = torch.empty(max(self.nMeshes, 4), dtype=torch.int32, device=dev)
        self.mesh_aabbs = torch.empty((self.nMeshes, 6), dtype=torch.float32, device=dev)
        self.rays = self.ray_offsets = self.hits = None
        self.nRays = 0
        self._desc = _Batch()
        d = self._desc
        d.dTriangles, d.dMeshTriangleOffsets = _ptr(triangles), _ptr(tri_offsets)
        d.nMeshes, d.nTriangles, d.buildOption = self.nMeshes, self.nTriangles, int(buildOption)
        d.dInternals, d.dRootNodes, d.dMeshAABBs = _ptr(self.internals), _ptr(self.roots), _ptr(self.mesh_aabbs)
        d.dScratch, d.scratchBytes = _ptr(self.scratch), self.scratch.numel()
        self._graphs = []

    def set_rays(self, rays, ray_offsets, rayQuery: int = RAY_QUERY_CLOSEST, hits=None):
        """Rays float32 (nRays, 8) (ro.xyz, tmin, rd.xyz, tmax), mesh after
        mesh; ray_offsets (nMeshes + 1, int32 on the device)."""
        import torch
        _require_cuda(rays, "rays")
        _require_cuda(ray_offsets, "ray_offsets")
        self.rays, self.ray_offsets, self.nRays = rays, ray_offsets, rays.numel() // 8
        if hits is None:
            hits = torch.empty((max(self.nRays, 1), 8), dtype=torch.int32, device=rays.device)
        self.hits = hits
        d = self._desc
        d.dRays, d.dMeshRayOffsets, d.nRays, d.rayQuery, d.dHits = (_ptr(rays), _ptr(ray_offsets), self.nRays,
                                                                    int(rayQuery), _ptr(hits))
        return self

    def build(self, params: BatchParams | None = None, stream=None):
        _check(lib().mlbvh_build_batched(ctypes.byref(self._desc), None if params is None else ctypes.byref(params),
                                         _stream(stream)))
        return self

    def trace(self, params: BatchParams | None = None, stream=None):
        _check(lib().mlbvh_trace_batched(ctypes.byref(self._desc), None if params is None else ctypes.byref(params),
                                         _stream(stream)))
        return self.hits

    def status(self, stream=None) -> None:
        """Synchronise; raise on bad offsets or a bounded wait that gave up."""
        _check(lib().mlbvh_scratch_status(_ptr(self.scratch), _stream(stream)))

    def autotune(self, stream=None):
        """Returns (BatchParams, build ms, trace ms) of the fastest candidates."""
        p = BatchParams()
        b, t = ctypes.c_float(0), ctypes.c_float(0)
        _check(lib().mlbvh_batch_autotune(ctypes.byref(self._desc), ctypes.byref(p), ctypes.byref(b),
                                          ctypes.byref(t), _stream(stream)))
        return p, b.value, t.value

    def graph(self, params: BatchParams | None = None, stages: int = 3) -> "BatchGraph":
        g = _vp()
        _check(lib().mlbvh_batch_graph_create(ctypes.byref(self._desc),
                                              None if params is None else ctypes.byref(params), int(stages),
                                              ctypes.byref(g)))
        return BatchGraph(g)

    def mesh_nodes(self, m: int, offsets_host) -> tuple:
        """(node rows, triangle range) of mesh m given the host offsets."""
        a, b = int(offsets_host[m]), int(offsets_host[m + 1])
        return self.internals[a - m: b - m - 1], (a, b)


class BatchGraph:
    """A CUDA graph of a batch's build and/or traversal."""

    def __init__(self, handle):
        self._h = handle

    def launch(self, stream=None):
        _check(lib().mlbvh_batch_graph_launch(self._h, _stream(stream)))

    def close(self):
        if self._h:
            lib().mlbvh_batch_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_obj(path: str):
    """mlbvh_obj_load: (triangles float32 (n, 9), attributes float32 (n, 15)
    as TriangleAttrib: shading normals, reflectance, emissive), host arrays."""
    L = lib()
    h = _vp()
    _check(L.mlbvh_obj_load(os.fsencode(path), ctypes.byref(h)))
    try:
        n = L.mlbvh_obj_triangle_count(h)
        if n == 0:
            return np.zeros((0, 9), np.float32), np.zeros((0, 15), np.float32)
        tp = ctypes.cast(L.mlbvh_obj_triangles(h), ctypes.POINTER(ctypes.c_float))
        ap = ctypes.cast(L.mlbvh_obj_attribs(h), ctypes.POINTER(ctypes.c_float))
        tris = np.ctypeslib.as_array(tp, shape=(n, 9)).copy()
        attribs = np.ctypeslib.as_array(ap, shape=(n, 15)).copy()
    finally:
        L.mlbvh_obj_free(h)
    return tris, attribs
