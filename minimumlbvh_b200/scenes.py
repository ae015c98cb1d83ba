"""Seeded synthetic scenes and rays for the MinimumLBVH workloads.

The reference renders one OBJ asset through a window; the workloads measured
here are synthetic and fully determined by their seed (numpy PCG64):

* ``heightfield_icospheres`` — 212,992 triangles: a 256 x 256-quad heightfield
  over [-1, 1]^2 (x, z) whose height y is a sum of 4 sine octaves (amplitude
  0.1 halving per octave, frequency 2^k * 2*pi, seeded phase and direction),
  plus 64 level-3 icospheres (1,280 triangles each) of radius U[0.02, 0.1],
  placed uniformly above the field with a uniformly random rotation.
* ``gaussian_soup`` — n triangles in 64 Gaussian clusters (centres uniform in
  the unit cube, sigma 0.02); each triangle is equilateral with a lognormal
  edge length (median 0.004, sigma 0.5) and a uniformly random orientation.

* ``batched_soup`` — the batched workload: meshes with triangle counts
  log-uniform in [lo, hi], each a Gaussian-cluster soup as above in its own
  unit box, laid out back to back; ``batched_rays`` gives every mesh a
  log-uniform number of rays with origins uniform in the mesh's bounding box
  expanded by 10% and directions uniform on the sphere. Both are generated
  with torch (seeded generator on the given device), so the 32M-triangle
  batch can be made directly in device memory.

Triangle arrays are float32 of shape (n, 9): v0.xyz, v1.xyz, v2.xyz per
triangle, the byte layout of minimum_lbvh::Triangle.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "heightfield_icospheres",
    "gaussian_soup",
    "icosphere",
    "random_rays",
    "camera_heightfield",
    "camera_soup",
    "pt_attributes",
    "quad_light",
    "diff_scene",
    "albedo",
    "log_uniform_counts",
    "batched_soup",
    "batched_rays",
    "camera_rays",
]


def _rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """n uniformly random rotation matrices (unit quaternions from 4 normals)."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - z * w)
    r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w)
    r[:, 2, 1] = 2 * (y * z + x * w)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def icosphere(level: int = 3) -> np.ndarray:
    """Unit icosphere by repeated 4:1 subdivision of an icosahedron.

    Returns (20 * 4**level, 3, 3) float64 triangle corners (outward winding).
    """
    t = (1.0 + 5.0**0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    tri = v[np.array(faces)]
    for _ in range(level):
        a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tri = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                              np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)])
    return tri


def heightfield_icospheres(seed: int = 0, quads: int = 256, spheres: int = 64, level: int = 3) -> np.ndarray:
    """The 212,992-triangle heightfield + icospheres scene (see module doc)."""
    rng = np.random.default_rng(seed)
    phase = rng.uniform(0.0, 2.0 * np.pi, 4)
    angle = rng.uniform(0.0, 2.0 * np.pi, 4)
    g = np.linspace(-1.0, 1.0, quads + 1)
    x, z = np.meshgrid(g, g, indexing="xy")
    y = np.zeros_like(x)
    for k in range(4):
        d = x * np.cos(angle[k]) + z * np.sin(angle[k])
        y += 0.1 * 2.0**-k * np.sin(2.0**k * 2.0 * np.pi * d + phase[k])
    p = np.stack([x, y, z], -1)  # (quads+1, quads+1, 3)
    p00, p10, p01, p11 = p[:-1, :-1], p[:-1, 1:], p[1:, :-1], p[1:, 1:]
    t0 = np.stack([p00, p01, p10], 2).reshape(-1, 3, 3)
    t1 = np.stack([p10, p01, p11], 2).reshape(-1, 3, 3)
    field = np.stack([t0, t1], 1).reshape(-1, 3, 3)
    unit = icosphere(level)
    radius = rng.uniform(0.02, 0.1, spheres)
    centre = np.stack([rng.uniform(-0.9, 0.9, spheres), rng.uniform(0.25, 0.6, spheres),
                       rng.uniform(-0.9, 0.9, spheres)], -1)
    rot = _rotations(rng, spheres)
    balls = np.einsum("sij,tvj->stvi", rot, unit) * radius[:, None, None, None] + centre[:, None, None, :]
    tris = np.concatenate([field, balls.reshape(-1, 3, 3)])
    return np.ascontiguousarray(tris.reshape(-1, 9).astype(np.float32))


def gaussian_soup(n: int = 4_194_304, clusters: int = 64, sigma: float = 0.02, seed: int = 1,
                  median_edge: float = 0.004, edge_sigma: float = 0.5) -> np.ndarray:
    """n equilateral triangles in Gaussian clusters (see module doc)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, (clusters, 3))
    out = np.empty((n, 9), dtype=np.float32)
    base = np.array([[1.0, 0.0, 0.0], [-0.5, 0.75**0.5, 0.0], [-0.5, -(0.75**0.5), 0.0]]) / 3.0**0.5
    chunk = 1 << 20
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        cid = (np.arange(s, s + m) % clusters)
        c = centres[cid] + rng.normal(0.0, sigma, (m, 3))
        edge = np.exp(np.log(median_edge) + edge_sigma * rng.standard_normal(m))
        rot = _rotations(rng, m)
        v = np.einsum("mij,vj->mvi", rot, base) * edge[:, None, None] + c[:, None, :]
        out[s:s + m] = v.reshape(m, 9)
    return out


def random_rays(n: int, lo, hi, seed: int = 2, tmax: float = 3.402823466e38) -> np.ndarray:
    """n rays (float32 (n, 8): ro.xyz, tmin=0, rd.xyz, tmax) with origins uniform
    in the box [lo, hi] expanded by 10% and directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    ext = (hi - lo) * 0.1
    ro = rng.uniform(lo - ext, hi + ext, (n, 3))
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), dtype=np.float32)
    rays[:, 0:3] = ro
    rays[:, 4:7] = d
    rays[:, 7] = np.float32(tmax)
    return rays


# Cameras of the two single-mesh workloads: (eye, center, up, fovy radians).
def camera_heightfield():
    """Eye above the heightfield looking down at 45 degrees."""
    return (0.0, 1.6, 1.6), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), np.float32(np.deg2rad(45.0))


def camera_soup():
    """Eye in front of the unit cube holding the Gaussian soup."""
    return (0.5, 0.5, -1.2), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), np.float32(np.deg2rad(40.0))


def pt_attributes(n: int, seed: int = 3, light_fraction: float = 0.002) -> np.ndarray:
    """Per-triangle TriangleAttrib records (float32 (n, 15)): shading normals
    (unused by pt), reflectance uniform in [0.1, 0.9]^3, and a small random
    subset of emitters with radiance 10."""
    rng = np.random.default_rng(seed)
    a = np.zeros((n, 15), dtype=np.float32)
    a[:, 9:12] = rng.uniform(0.1, 0.9, (n, 3))
    emit = rng.random(n) < light_fraction
    a[emit, 12:15] = 10.0
    return a


def quad_light(y: float = 1.4, half: float = 0.25) -> np.ndarray:
    """A 0.5 x 0.5 horizontal quad (two triangles) centred above the
    heightfield at height y: float32 (2, 9)."""
    a, b, c, d = (-half, y, -half), (half, y, -half), (half, y, half), (-half, y, half)
    return np.array([a + b + c, a + c + d], dtype=np.float32)


def diff_scene(seed: int = 0, albedo_seed: int = 1, light_radiance: float = 10.0):
    """The differentiable-rendering scene: the 212,992-triangle heightfield +
    icospheres with a quad light of radiance 10 appended (212,994 triangles),
    per-triangle grey albedo uniform in [0.1, 0.9] (seeded) and emission
    (light_radiance on the two light triangles, 0 elsewhere)."""
    tris = np.concatenate([heightfield_icospheres(seed), quad_light()])
    emission = np.zeros(len(tris), np.float32)
    emission[-2:] = light_radiance
    return tris, albedo(len(tris), albedo_seed), emission


def albedo(n: int, seed: int) -> np.ndarray:
    """Per-triangle grey albedo uniform in [0.1, 0.9] (float32)."""
    return np.random.default_rng(seed).uniform(0.1, 0.9, n).astype(np.float32)


def log_uniform_counts(n: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """n integers log-uniform in [lo, hi] (int64)."""
    rng = np.random.default_rng(seed)
    c = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    return np.clip(np.rint(c), lo, hi).astype(np.int64)


def _soup_torch(counts, clusters: int, sigma: float, median_edge: float, edge_sigma: float, gen, device):
    """Gaussian-cluster soups (see gaussian_soup) for every mesh of ``counts``,
    back to back, generated with torch: float32 tensor (sum(counts), 9)."""
    import torch
    nm = len(counts)
    n = int(np.sum(counts))
    mesh = torch.repeat_interleave(torch.arange(nm, device=device),
                                   torch.as_tensor(np.asarray(counts), device=device))
    starts = torch.as_tensor(np.concatenate([[0], np.cumsum(counts)[:-1]]), device=device)
    local = torch.arange(n, device=device) - starts[mesh]
    centres = torch.rand((nm, clusters, 3), generator=gen, device=device, dtype=torch.float64)
    out = torch.empty((n, 9), dtype=torch.float32, device=device)
    base = torch.tensor([[1.0, 0.0, 0.0], [-0.5, 0.75**0.5, 0.0], [-0.5, -(0.75**0.5), 0.0]],
                        dtype=torch.float64, device=device) / 3.0**0.5
    chunk = 1 << 22
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        c = centres[mesh[s:e], local[s:e] % clusters] + sigma * torch.randn((m, 3), generator=gen, device=device,
                                                                          dtype=torch.float64)
        edge = torch.exp(np.log(median_edge) + edge_sigma * torch.randn(m, generator=gen, device=device,
                                                                        dtype=torch.float64))
        q = torch.randn((m, 4), generator=gen, device=device, dtype=torch.float64)
        q = q / q.norm(dim=1, keepdim=True)
        w, x, y, z = q.unbind(1)
        r = torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                         2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                         2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1).view(m, 3, 3)
        v = torch.einsum("mij,vj->mvi", r, base) * edge[:, None, None] + c[:, None, :]
        out[s:e] = v.reshape(m, 9).to(torch.float32)
    return out


def batched_soup(n_meshes: int = 1024, lo: int = 64, hi: int = 262_144, seed: int = 7, device="cpu",
                 clusters: int = 64, sigma: float = 0.02, median_edge: float = 0.004, edge_sigma: float = 0.5):
    """The batched workload's meshes (see module doc). Returns (triangles
    float32 tensor (n, 9) on ``device``, triangle offsets int64 numpy array of
    n_meshes + 1)."""
    import torch
    counts = log_uniform_counts(n_meshes, lo, hi, seed)
    gen = torch.Generator(device=device).manual_seed(seed)
    tris = _soup_torch(counts, clusters, sigma, median_edge, edge_sigma, gen, device)
    return tris, np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def batched_rays(tris, tri_offsets: np.ndarray, lo: int = 4096, hi: int = 1_048_576, seed: int = 8, counts=None,
                 tmax: float = 3.402823466e38):
    """Rays of the batched workload: mesh m gets counts[m] rays (log-uniform
    in [lo, hi] unless given) with origins uniform in its bounding box
    expanded by 10% and directions uniform on the sphere. Returns (rays
    float32 tensor (R, 8) on the triangles' device, ray offsets int64 numpy
    array of n_meshes + 1)."""
    import torch
    device = tris.device
    nm = len(tri_offsets) - 1
    if counts is None:
        counts = log_uniform_counts(nm, lo, hi, seed)
    counts = np.asarray(counts, np.int64)
    tmesh = torch.repeat_interleave(torch.arange(nm, device=device),
                                    torch.as_tensor(np.diff(tri_offsets), device=device))
    pts = tris.view(-1, 3, 3)
    bmin = torch.full((nm, 3), float("inf"), device=device).scatter_reduce(
        0, tmesh[:, None].expand(-1, 3), pts.amin(1), "amin")
    bmax = torch.full((nm, 3), float("-inf"), device=device).scatter_reduce(
        0, tmesh[:, None].expand(-1, 3), pts.amax(1), "amax")
    rmesh = torch.repeat_interleave(torch.arange(nm, device=device), torch.as_tensor(counts, device=device))
    gen = torch.Generator(device=device).manual_seed(seed)
    n = int(counts.sum())
    rays = torch.zeros((n, 8), dtype=torch.float32, device=device)
    chunk = 1 << 24
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lo3, hi3 = bmin[rmesh[s:e]].double(), bmax[rmesh[s:e]].double()
        ext = (hi3 - lo3) * 0.1
        u = torch.rand((e - s, 3), generator=gen, device=device, dtype=torch.float64)
        rays[s:e, 0:3] = (lo3 - ext + u * (hi3 - lo3 + 2 * ext)).float()
        d = torch.randn((e - s, 3), generator=gen, device=device, dtype=torch.float64)
        rays[s:e, 4:7] = (d / d.norm(dim=1, keepdim=True)).float()
    rays[:, 7] = float(np.float32(tmax))
    return rays, np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def camera_rays(origin, right, up, w: int, h: int, step: int = 2) -> np.ndarray:
    """Pinhole rays (RayGenerator::shoot, camera.h:24-31, in FP64 numpy) of
    every `step`-th pixel of a w x h frame: float32 (n, 8) with tmin 0 and
    tmax FLT_MAX."""
    o, right, up = (np.asarray(x, np.float64) for x in (origin, right, up))
    fwd = np.cross(up, right)
    fwd /= np.linalg.norm(fwd)
    ys, xs = np.divmod(np.arange(0, w * h, step), w)
    u, v = (xs / w)[:, None], (ys / h)[:, None]
    to = o + fwd + (-right + u * 2 * right) + (up - v * 2 * up)
    rays = np.zeros((len(xs), 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = to - o
    rays[:, 7] = np.float32(3.402823466e38)
    return rays
