"""FP64 check of hit distances (host, numpy).

For a hit of ray (ro, rd) on triangle (v0, v1, v2) the reference computes, in
FP32, t = dot(v0 - ro, ng) / dot(ng, rd) with ng = cross(v1 - v0, v2 - v1)
(intersectRayTriangle, minimum_lbvh.h:363-413). `fp64_t` evaluates the same
formula in FP64. `t_error_bound` is a forward error bound of the FP32
evaluation, relative to |t|: with u = 2^-24,

    |t32 - t64| <= u * (4 kN + 4 kD + 2) * |t64|,

where kN = (sum |a_i| (|ng_i| + c_i)) / |N| and kD = (sum |rd_i| (|ng_i| +
c_i)) / |D| are the condition numbers of the numerator N (a = v0 - ro) and the
denominator D, and c_i = |e0_j e1_k| + |e0_k e1_j| bounds the rounding of the
cross product component i. Near-grazing hits (D near 0) get large bounds, as
they should.
"""
from __future__ import annotations

import numpy as np


def _tri_parts(tris, idx):
    t = np.asarray(tris, np.float32).reshape(-1, 3, 3)[idx].astype(np.float64)
    return t[:, 0], t[:, 1], t[:, 2]


def fp64_t(tris, rays, tri_index):
    """FP64 ray-plane distances for rays (n, 8) and hit triangle indices (n,)."""
    v0, v1, v2 = _tri_parts(tris, tri_index)
    ro = rays[:, 0:3].astype(np.float64)
    rd = rays[:, 4:7].astype(np.float64)
    ng = np.cross(v1 - v0, v2 - v1)
    return np.einsum("ij,ij->i", v0 - ro, ng) / np.einsum("ij,ij->i", ng, rd)


def t_error_bound(tris, rays, tri_index):
    """The relative bound above, per hit (multiply by |t64|)."""
    v0, v1, v2 = _tri_parts(tris, tri_index)
    ro = rays[:, 0:3].astype(np.float64)
    rd = rays[:, 4:7].astype(np.float64)
    e0, e1 = v1 - v0, v2 - v1
    ng = np.cross(e0, e1)
    c = np.stack([np.abs(e0[:, 1] * e1[:, 2]) + np.abs(e0[:, 2] * e1[:, 1]),
                  np.abs(e0[:, 2] * e1[:, 0]) + np.abs(e0[:, 0] * e1[:, 2]),
                  np.abs(e0[:, 0] * e1[:, 1]) + np.abs(e0[:, 1] * e1[:, 0])], 1)
    a = v0 - ro
    N = np.einsum("ij,ij->i", a, ng)
    D = np.einsum("ij,ij->i", ng, rd)
    with np.errstate(divide="ignore", invalid="ignore"):
        kN = np.einsum("ij,ij->i", np.abs(a), np.abs(ng) + c) / np.abs(N)
        kD = np.einsum("ij,ij->i", np.abs(rd), np.abs(ng) + c) / np.abs(D)
    return 2.0**-24 * (4 * kN + 4 * kD + 2)


def check_hits(tris, rays, hits_u32):
    """For Hit records (n, 8) as uint32: FP64 comparison of every hit's t.
    Returns dict(hits, max_abs_err, max_rel_err, max_bound_ratio) where the
    bound ratio is |t32 - t64| / (bound * |t64|) (<= 1 within the bound)."""
    hit = hits_u32[:, 7] != 0xFFFFFFFF
    idx = hits_u32[hit, 7].astype(np.int64)
    r = np.asarray(rays)[hit]
    t32 = hits_u32[hit, 0].view(np.float32).astype(np.float64)
    t64 = fp64_t(tris, r, idx)
    err = np.abs(t32 - t64)
    rel = err / np.maximum(np.abs(t64), 1e-300)
    bound = t_error_bound(tris, r, idx)
    ratio = rel / bound
    return {"hits": int(hit.sum()), "max_abs_err": float(err.max(initial=0.0)),
            "max_rel_err": float(rel.max(initial=0.0)), "max_bound_ratio": float(np.nanmax(ratio, initial=0.0))}
