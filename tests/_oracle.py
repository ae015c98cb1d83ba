"""ctypes access to the checkers: oracle/liboracle.so (the restatement) and
oracle/_ref/libmlbvh_ref.so (the reference's own CPU code, when built).

Test infrastructure only. Builds liboracle.so with gcc on first use if it is
missing (gcc is the only requirement); the reference library cannot be
rebuilt without the reference sources and is optional.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libmlbvh_ref.so")

_vp = ctypes.c_void_p
_u32, _i32, _f32, _u64 = ctypes.c_uint32, ctypes.c_int, ctypes.c_float, ctypes.c_uint64

FLT_MAX = np.float32(3.402823466e38)
LEAF = 0x80000000
INVALID = 0x7FFFFFFF


class F3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


def P(a):
    return None if a is None else a.ctypes.data_as(_vp)


_oracle = None
_ref = None


def oracle() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        src = os.path.join(ORACLE_DIR, "mlbvh_oracle.c")
        if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(src):
            subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True, capture_output=True)
        L = ctypes.CDLL(ORACLE_LIB)
        sig = {
            "orc_version": (_i32, []),
            "orc_set_threads": (None, [_i32]),
            "orc_clz": (_i32, [_u32]), "orc_clz64": (_i32, [_u64]), "orc_ffs": (_i32, [_u32]),
            "orc_ffs64": (_i32, [_u64]), "orc_delta": (_i32, [_u32, _u32]),
            "orc_splat3": (_u64, [_u32]), "orc_compact3": (_u32, [_u64]),
            "orc_encode_morton": (_u64, [_u32, _u32, _u32]), "orc_encode_morton_naive": (_u64, [_u32, _u32, _u32]),
            "orc_decode_morton": (None, [_u64, _vp, _vp, _vp]),
            "orc_scene_aabb": (None, [_vp, _u32, _vp]),
            "orc_morton_keys": (None, [_vp, _u32, _u32, _vp, _vp]),
            "orc_sort_pairs": (None, [_vp, _vp, _u32]),
            "orc_build": (_i32, [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_build_from_keys": (_i32, [_vp, _vp, _vp, _u32, _vp, _vp, _vp]),
            "orc_validate": (_i32, [_vp, _vp, _u32, _u32, _i32]),
            "orc_check_tree": (_i32, [_vp, _vp, _u32, _u32]),
            "orc_build_ploc": (_i32, [_vp, _u32, _u32, _i32, _vp, _vp]),
            "orc_sah_cost": (ctypes.c_double, [_vp, _u32, _u32]),
            "orc_trace": (None, [_vp, _vp, _u32, _vp, _u32, _i32, _i32, _vp, _vp, _vp]),
            "orc_trace_replay": (None, [_vp, _vp, _u32, _vp, _u32, _i32, _i32, _vp, _vp, _vp]),
            "orc_build_wide": (None, [_vp, _u32, _vp]),
            "orc_trace_wide": (None, [_vp, _vp, _vp, _u32, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _i32]),
            "orc_quantise_wide": (_i32, [_vp, _u32, _vp]),
            "orc_fma_dir": (_f32, [_f32, _f32, _f32, _i32]),
            "orc_trace_wide_quantised": (None, [_vp, _i32, _vp, _vp, _u32, _u32, _vp, _u32, _vp, _vp, _vp, _vp,
                                                _i32]),
            "orc_lookat": (None, [F3, F3, F3, _f32, _i32, _i32, _vp]),
            "orc_sobol": (None, [_u32, _u32, _u32, _u32, _vp, _vp]),
            "orc_hash_pcg": (_u32, [_u32]),
            "orc_sincos": (None, [_f32, _vp, _vp]),
            "orc_render_ao": (None, [_vp, _vp, _i32, _i32, _vp, _u32, _vp, _vp, _i32, _i32, _f32, _u32, _i32,
                                     _i32, _i32, _vp]),
            "orc_render_pt": (None, [_vp, _i32, _i32, _vp, _u32, _vp, _vp, _vp, _i32, _i32, _i32, _i32]),
            "orc_pack": (None, [_vp, _vp, _i32]),
            "orc_render_normal": (None, [_vp, _i32, _i32, _vp, _u32, _vp, _vp]),
            "orc_quantise": (_i32, [_vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp]),
            "orc_check_quantised": (_i32, [_vp, _u32, _vp, _vp]),
            "orc_trace_quantised": (None, [_vp, _vp, _vp, _vp, _vp, _u32, _i32, _vp, _vp, _vp, _vp]),
            "orc_trace_quantised_replay": (None, [_vp, _vp, _vp, _vp, _vp, _u32, _i32, _i32, _vp, _vp, _vp, _vp]),
            "orc_pt_diff_render": (None, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_pt_diff_adjoint": (None, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _u32, _vp, _vp, _vp, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _oracle = L
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_LIB)
        sig = {
            "ref_version": (_i32, []), "ref_threads": (_i32, []),
            "ref_cpu_builder": (None, [_vp, _i32, _u32, _vp, _vp, _vp]),
            "ref_build_stable": (None, [_vp, _i32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _i32]),
            "ref_toy_tree": (None, [_vp, _i32, _vp, _vp, _vp]),
            "ref_trace": (None, [_vp, _vp, _u32, _vp, _i32, _i32, _i32, _vp]),
            "ref_lookat": (None, [_vp, _vp, _vp, _f32, _i32, _i32, _vp]),
            "ref_shoot": (None, [_vp, _i32, _i32, _i32, _i32, _vp, _vp]),
            "ref_ao": (None, [_vp, _i32, _i32, _vp, _u32, _vp, _vp, _i32]),
            "ref_ao_param": (None, [_vp, _i32, _i32, _vp, _u32, _vp, _vp, _i32, _f32, _u32, _i32, _i32, _vp]),
            "ref_normal": (None, [_vp, _i32, _i32, _vp, _u32, _vp, _vp]),
            "ref_pt": (None, [_vp, _vp, _i32, _i32, _vp, _u32, _vp, _vp, _vp, _i32, _i32]),
            "ref_pack": (None, [_vp, _vp, _i32]),
            "ref_sobol": (None, [_u32, _u32, _u32, _u32, _vp]),
            "ref_splat3": (_u64, [_u32]), "ref_compact3": (_u32, [_u64]),
            "ref_encode_morton": (_u64, [_u32, _u32, _u32]), "ref_encode_morton_naive": (_u64, [_u32, _u32, _u32]),
            "ref_clz": (_i32, [_u32]), "ref_clz64": (_i32, [_u64]), "ref_ffs": (_i32, [_u32]),
            "ref_ffs64": (_i32, [_u64]), "ref_hash_pcg": (_u32, [_u32]),
            "ref_aabb_morton": (_u64, [_vp, _vp, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref = L
    return _ref


# ------------------------------------------------------------ oracle wrappers
def build(tris: np.ndarray, option: int = 0):
    """Oracle build: dict of nodes (n-1, 16) u32, deltas, root, keys, indices, scene."""
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = tris.shape[0]
    nodes = np.zeros((max(n - 1, 1), 16), np.uint32)
    deltas = np.zeros(max(n - 1, 1), np.uint8)
    root = np.zeros(1, np.uint32)
    keys = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    scene = np.zeros(6, np.float32)
    rc = oracle().orc_build(P(tris), n, option, P(nodes), P(deltas), P(root), P(keys), P(idx), P(scene))
    assert rc == 0
    return dict(nodes=nodes[: n - 1], deltas=deltas[: n - 1], root=int(root[0]), keys=keys, indices=idx, scene=scene)


def build_ploc(tris: np.ndarray, option: int = 0, radius: int = 8):
    """Oracle PLOC build: dict of nodes (n-1, 16) u32 (in-order numbering),
    root and the number of clustering iterations."""
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = tris.shape[0]
    nodes = np.zeros((max(n - 1, 1), 16), np.uint32)
    root = np.zeros(1, np.uint32)
    it = oracle().orc_build_ploc(P(tris), n, option, radius, P(nodes), P(root))
    assert it >= 0
    return dict(nodes=nodes[: n - 1], root=int(root[0]), iterations=it)


def sah_cost(nodes, root: int) -> float:
    nodes = np.ascontiguousarray(nodes, np.uint32).reshape(-1, 16)
    return float(oracle().orc_sah_cost(P(nodes), nodes.shape[0] + 1, root))


def check_tree(nodes, tris, root: int) -> bool:
    nodes = np.ascontiguousarray(nodes, np.uint32).reshape(-1, 16)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    return bool(oracle().orc_check_tree(P(nodes), P(tris), tris.shape[0], root))


def ref_build(tris: np.ndarray, option: int = 0, parallel: int = 0):
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = tris.shape[0]
    nodes = np.zeros((max(n - 1, 1), 16), np.uint32)
    deltas = np.zeros(max(n - 1, 1), np.uint8)
    root = np.zeros(1, np.uint32)
    keys = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    scene = np.zeros(6, np.float32)
    ref().ref_build_stable(P(tris), n, option, P(nodes), P(deltas), P(root), P(keys), P(idx), P(scene), parallel)
    return dict(nodes=nodes[: n - 1], deltas=deltas[: n - 1], root=int(root[0]), keys=keys, indices=idx, scene=scene)


def trace(nodes, tris, root, rays, query=0, mode=0, counters=False):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 8), np.uint32)
    nv = np.zeros(n, np.uint32) if counters else None
    nt = np.zeros(n, np.uint32) if counters else None
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    oracle().orc_trace(P(nodes_c), P(np.ascontiguousarray(tris, np.float32)), root, P(rays), n, query, mode,
                       P(hits), P(nv), P(nt))
    if counters:
        return hits, nv, nt
    return hits


def trace_replay(nodes, tris, root, rays, query=0, depth=16, counters=False):
    """The replay walk over the reference node layout (same hits as trace
    mode 0, fewer node visits)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 8), np.uint32)
    nv = np.zeros(n, np.uint32) if counters else None
    nt = np.zeros(n, np.uint32) if counters else None
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    oracle().orc_trace_replay(P(nodes_c), P(np.ascontiguousarray(tris, np.float32)), root, P(rays), n, query, depth,
                              P(hits), P(nv), P(nt))
    if counters:
        return hits, nv, nt
    return hits


def build_wide(nodes, n):
    """The 4-wide tree of a built tree: (n - 1, 32) uint32 slots."""
    out = np.zeros((max(n - 1, 0), 32), np.uint32)
    if n > 1:
        oracle().orc_build_wide(P(np.ascontiguousarray(nodes, np.uint32)), n, P(out))
    return out


def trace_wide(wide, nodes, tris, root, rays, query=1):
    """Rays over the 4-wide tree (query 1 any-hit, 0 closest-hit): hits and
    per-ray (visits, tests, restarts)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n, m = len(tris), rays.shape[0]
    hits = np.zeros((m, 8), np.uint32)
    nv, nt, nr = (np.zeros(m, np.uint32) for _ in range(3))
    wide_c = np.ascontiguousarray(wide, np.uint32) if len(wide) else np.zeros((1, 32), np.uint32)
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    oracle().orc_trace_wide(P(wide_c), P(nodes_c), P(tris), n, root, P(rays), m, P(hits), P(nv), P(nt), P(nr),
                            query)
    return hits, nv, nt, nr


def quantise_wide(wide, n):
    """Quantised slots of a 4-wide tree: ((n - 1, 16) uint32, all quantised?)."""
    out = np.zeros((max(n - 1, 0), 16), np.uint32)
    ok = 1
    if n > 1:
        ok = oracle().orc_quantise_wide(P(np.ascontiguousarray(wide, np.uint32)), n, P(out))
    return out, bool(ok)


def trace_wide_quantised(qwide, nodes, tris, root, rays, fallback=False, query=1):
    """Rays over quantised wide slots (query 1 any-hit, 0 closest-hit): hits,
    visits, tests, restarts."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n, m = len(tris), rays.shape[0]
    hits = np.zeros((m, 8), np.uint32)
    nv, nt, nr = (np.zeros(m, np.uint32) for _ in range(3))
    q_c = np.ascontiguousarray(qwide, np.uint32) if len(qwide) else np.zeros((1, 16), np.uint32)
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    oracle().orc_trace_wide_quantised(P(q_c), int(fallback), P(nodes_c), P(tris), n, root, P(rays), m, P(hits),
                                      P(nv), P(nt), P(nr), query)
    return hits, nv, nt, nr


def ref_trace(nodes, tris, root, rays, query=0, mode=0):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 8), np.uint32)
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    ref().ref_trace(P(nodes_c), P(np.ascontiguousarray(tris, np.float32)), root, P(rays), n, query, mode, P(hits))
    return hits


def lookat(eye, center, up, fovy, w, h) -> np.ndarray:
    cam = np.zeros(9, np.float32)
    oracle().orc_lookat(F3(*eye), F3(*center), F3(*up), float(fovy), w, h, P(cam))
    return cam


def render_ao(cam, root, nodes, tris, w, h, n_samples=16, radius=1.0, seed=12345, use_sobol=1, trig=1,
              rows=None, counters=False):
    pixels = np.zeros(w * h, np.uint32)
    occ = np.zeros(w * h, np.uint32)
    cnt = np.zeros(3, np.uint64)
    rb, re = (0, h) if rows is None else rows
    nodes_c = np.ascontiguousarray(nodes, np.uint32) if len(nodes) else np.zeros((1, 16), np.uint32)
    oracle().orc_render_ao(P(pixels), P(occ), w, h, P(np.ascontiguousarray(cam, np.float32)), root, P(nodes_c),
                           P(np.ascontiguousarray(tris, np.float32)), use_sobol, n_samples, float(radius), seed,
                           trig, rb, re, P(cnt))
    if counters:
        return pixels, occ, cnt
    return pixels, occ


def ref_ao(cam, root, nodes, tris, w, h, use_sobol=1):
    pixels = np.zeros(w * h, np.uint32)
    ref().ref_ao(P(pixels), w, h, P(np.ascontiguousarray(cam, np.float32)), root,
                 P(np.ascontiguousarray(nodes, np.uint32)), P(np.ascontiguousarray(tris, np.float32)), use_sobol)
    return pixels


def render_pt(accum, cam, root, nodes, tris, attribs, w, h, use_sobol=1, max_spp=1 << 30, max_depth=1024, trig=1):
    oracle().orc_render_pt(P(accum), w, h, P(np.ascontiguousarray(cam, np.float32)), root,
                           P(np.ascontiguousarray(nodes, np.uint32)), P(np.ascontiguousarray(tris, np.float32)),
                           P(np.ascontiguousarray(attribs, np.float32)), use_sobol, max_spp, max_depth, trig)
    return accum


def ref_pt(accum, cam, root, nodes, tris, attribs, w, h, use_sobol=1, max_spp=1 << 30):
    pixels = np.zeros(w * h, np.uint32)
    ref().ref_pt(P(pixels), P(accum), w, h, P(np.ascontiguousarray(cam, np.float32)), root,
                 P(np.ascontiguousarray(nodes, np.uint32)), P(np.ascontiguousarray(tris, np.float32)),
                 P(np.ascontiguousarray(attribs, np.float32)), use_sobol, max_spp)
    return accum


def render_normal(cam, root, nodes, tris, w, h):
    pixels = np.zeros(w * h, np.uint32)
    oracle().orc_render_normal(P(pixels), w, h, P(np.ascontiguousarray(cam, np.float32)), root,
                               P(np.ascontiguousarray(nodes, np.uint32)), P(np.ascontiguousarray(tris, np.float32)))
    return pixels


def pack(accum, n):
    pixels = np.zeros(n, np.uint32)
    oracle().orc_pack(P(pixels), P(np.ascontiguousarray(accum, np.float32)), n)
    return pixels


def quantise(b: dict, tris: np.ndarray):
    """Oracle quantised tree of an oracle build: dict of qnodes (n-1, 8),
    parents (n-1,), qtris (n, 12) and header (4,), all uint32."""
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = len(tris)
    qn = np.zeros((max(n - 1, 1), 8), np.uint32)
    par = np.zeros(max(n - 1, 1), np.uint32)
    qt = np.zeros((n, 12), np.uint32)
    hd = np.zeros(4, np.uint32)
    nodes_c = np.ascontiguousarray(b["nodes"], np.uint32) if n > 1 else np.zeros((1, 16), np.uint32)
    oracle().orc_quantise(P(nodes_c), b["root"], P(tris), n, P(qn), P(par), P(qt), P(hd))
    return dict(qnodes=qn[: n - 1], parents=par[: n - 1], qtris=qt, header=hd)


def trace_quantised(q: dict, rays, query=0, counters=False, stack_depth=0):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 8), np.uint32)
    nv = np.zeros(n, np.uint32) if counters else None
    nt = np.zeros(n, np.uint32) if counters else None
    nu = np.zeros(n, np.uint32) if counters else None
    qn = q["qnodes"] if len(q["qnodes"]) else np.zeros((1, 8), np.uint32)
    par = q["parents"] if len(q["parents"]) else np.zeros(1, np.uint32)
    if stack_depth > 0:  # the replay walk with a stack of pending far children
        oracle().orc_trace_quantised_replay(P(np.ascontiguousarray(qn)), P(np.ascontiguousarray(par)),
                                            P(np.ascontiguousarray(q["qtris"])), P(q["header"]), P(rays), n, query,
                                            stack_depth, P(hits), P(nv), P(nt), P(nu))
    else:
        oracle().orc_trace_quantised(P(np.ascontiguousarray(qn)), P(np.ascontiguousarray(par)),
                                     P(np.ascontiguousarray(q["qtris"])), P(q["header"]), P(rays), n, query, P(hits),
                                     P(nv), P(nt), P(nu))
    if counters:
        return hits, nv, nt, nu
    return hits


def diff_render(b, tris, cam, w, h, spp, bounces, albedo, emission, fp64=False):
    """Oracle differentiable render: FP32 image (the kernel's, bit for bit) or
    FP64 image over the same path geometry."""
    img32 = None if fp64 else np.zeros(w * h, np.float32)
    img64 = np.zeros(w * h, np.float64) if fp64 else None
    oracle().orc_pt_diff_render(P(img32), P(img64), w, h, spp, bounces, P(np.ascontiguousarray(cam, np.float32)),
                                b["root"], P(np.ascontiguousarray(b["nodes"], np.uint32)),
                                P(np.ascontiguousarray(tris, np.float32)), P(np.ascontiguousarray(albedo, np.float32)),
                                P(np.ascontiguousarray(emission, np.float32)),
                                P(np.ascontiguousarray(albedo, np.float64)),
                                P(np.ascontiguousarray(emission, np.float64)))
    return img64 if fp64 else img32


def diff_adjoint(b, tris, cam, w, h, spp, bounces, albedo, emission, grad_image):
    """The FP64 host adjoint: dLoss/dAlbedo given dLoss/dImage."""
    grad = np.zeros(len(tris), np.float64)
    oracle().orc_pt_diff_adjoint(P(grad), P(np.ascontiguousarray(grad_image, np.float64)), w, h, spp, bounces,
                                 P(np.ascontiguousarray(cam, np.float32)), b["root"],
                                 P(np.ascontiguousarray(b["nodes"], np.uint32)), P(np.ascontiguousarray(tris, np.float32)),
                                 P(np.ascontiguousarray(albedo, np.float64)),
                                 P(np.ascontiguousarray(emission, np.float64)))
    return grad
