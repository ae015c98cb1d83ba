"""Generates the golden fixtures in this folder from the reference itself.

Every expected output here comes from oracle/_ref/libmlbvh_ref.so, i.e. the
reference's own minimum_lbvh.h / main_gpu.cu / sobol.h / camera.h compiled for
the host by oracle/Makefile (run `make -C oracle ref` first; it needs the
reference sources). Inputs are generated with minimumlbvh_b200.scenes and
stored next to the outputs, so the fixtures do not depend on the machine that
reads them.

    python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import _oracle as O  # noqa: E402
from minimumlbvh_b200 import scenes  # noqa: E402


def small_scene():
    """4,608 triangles: a 32 x 32-quad heightfield and 8 level-2 icospheres."""
    return scenes.heightfield_icospheres(seed=7, quads=32, spheres=8, level=2)


def main():
    R = O.ref()
    rng = np.random.default_rng(1234)

    # -- Morton / bit utilities (minimum_lbvh.h:99-195; unittest.cpp:10-105)
    xyz = rng.integers(0, 1 << 21, (4096, 3), dtype=np.uint64).astype(np.uint32)
    codes = np.array([R.ref_encode_morton(*map(int, v)) for v in xyz], np.uint64)
    sv = rng.integers(0, 1 << 32, 4096, dtype=np.uint64).astype(np.uint32)
    splat = np.array([R.ref_splat3(int(v)) for v in sv], np.uint64)
    lows = rng.uniform(-2, 0, (512, 3)).astype(np.float32)
    highs = (lows + rng.uniform(0.0, 3.0, (512, 3))).astype(np.float32)
    highs[:16, 0] = lows[:16, 0]  # degenerate axes: (p - lo) / 0
    pts = (lows + (highs - lows) * rng.uniform(-0.1, 1.1, (512, 3))).astype(np.float32)
    box_codes = np.array([R.ref_aabb_morton(O.P(lows[i]), O.P(highs[i]), O.P(pts[i])) for i in range(512)], np.uint64)
    clz_in = np.array([0] + [(0x80000000 >> i) | ((0x80000000 >> i) - 1) for i in range(32)] +
                      list(rng.integers(0, 1 << 32, 64, dtype=np.uint64)), np.uint64).astype(np.uint32)
    clz_out = np.array([R.ref_clz(int(v)) for v in clz_in], np.int32)
    ffs_out = np.array([R.ref_ffs(int(v)) for v in clz_in], np.int32)
    np.savez_compressed(os.path.join(HERE, "morton_kat.npz"), xyz=xyz, codes=codes, splat_in=sv, splat=splat,
                        box_lo=lows, box_hi=highs, box_p=pts, box_codes=box_codes, clz_in=clz_in, clz_out=clz_out,
                        ffs_out=ffs_out)

    # -- the toy tree of main.cpp:60-109
    toy = np.array([0b0010, 0b0011, 0b0100, 0b0101, 0b1000, 0b1100, 0b1101, 0b1111], np.uint32)
    tn = np.zeros((7, 16), np.uint32)
    td = np.zeros(7, np.uint8)
    tr = np.zeros(1, np.uint32)
    R.ref_toy_tree(O.P(toy), 8, O.P(tn), O.P(td), O.P(tr))
    np.savez_compressed(os.path.join(HERE, "toy_tree.npz"), keys=toy, nodes=tn, deltas=td, root=tr)

    # -- builds (BVHCPUBuilder::build with the stable key order)
    cases = {}
    for n in (1, 2, 3, 257, 4097):
        cases[f"soup{n}"] = (scenes.gaussian_soup(n, clusters=4, seed=100 + n), 0)
    cases["dup300"] = (np.tile(scenes.gaussian_soup(1, seed=5), (300, 1)), 0)
    cases["small_scene"] = (small_scene(), 0)
    cases["normal1000"] = (scenes.gaussian_soup(1000, clusters=2, seed=9), 1)
    out = {}
    for name, (tris, opt) in cases.items():
        b = O.ref_build(tris, opt)
        out[f"{name}/tris"] = tris
        out[f"{name}/option"] = np.array([opt], np.uint32)
        for k in ("nodes", "deltas", "keys", "indices", "scene"):
            out[f"{name}/{k}"] = b[k]
        out[f"{name}/root"] = np.array([b["root"]], np.uint32)
    np.savez_compressed(os.path.join(HERE, "builds.npz"), **out)

    # -- queries over the small scene
    tris = small_scene()
    b = O.ref_build(tris)
    rays = scenes.random_rays(4096, tris.reshape(-1, 3).min(0), tris.reshape(-1, 3).max(0), seed=11)
    short = rays.copy()
    short[::2, 7] = 0.05  # half the rays with a short far limit
    tr = {"rays": rays, "short_rays": short}
    for q, m in ((0, 0), (1, 0), (0, 1), (1, 1), (0, 2)):
        tr[f"hits_q{q}_m{m}"] = O.ref_trace(b["nodes"], tris, b["root"], rays, q, m)
        tr[f"short_q{q}_m{m}"] = O.ref_trace(b["nodes"], tris, b["root"], short, q, m)
    np.savez_compressed(os.path.join(HERE, "traces.npz"), **tr)

    # -- shading over the small scene (main_gpu.cu kernels run on the host)
    w, h = 64, 48
    eye, center, up, fovy = scenes.camera_heightfield()
    cam = np.zeros(9, np.float32)
    R.ref_lookat(O.P(np.array(eye, np.float32)), O.P(np.array(center, np.float32)), O.P(np.array(up, np.float32)),
                 float(fovy), w, h, O.P(cam))
    attribs = scenes.pt_attributes(len(tris), light_fraction=0.02)
    sh = {"camera": cam, "attribs": attribs, "size": np.array([w, h], np.int32)}
    sh["ao_sobol"] = O.ref_ao(cam, b["root"], b["nodes"], tris, w, h, 1)
    sh["ao_pcg"] = O.ref_ao(cam, b["root"], b["nodes"], tris, w, h, 0)
    normal = np.zeros(w * h, np.uint32)
    R.ref_normal(O.P(normal), w, h, O.P(cam), b["root"], O.P(b["nodes"]), O.P(tris))
    sh["normal"] = normal
    acc = np.zeros((w * h, 4), np.float32)
    for _ in range(2):
        O.ref_pt(acc, cam, b["root"], b["nodes"], tris, attribs, w, h, 1)
    sh["pt_sobol_2spp"] = acc.copy()
    px = np.zeros(w * h, np.uint32)
    R.ref_pack(O.P(px), O.P(acc), w * h)
    sh["pack"] = px
    acc = np.zeros((w * h, 4), np.float32)
    O.ref_pt(acc, cam, b["root"], b["nodes"], tris, attribs, w, h, 0)
    sh["pt_pcg_1spp"] = acc
    np.savez_compressed(os.path.join(HERE, "shading.npz"), **sh)

    # -- sample streams (sobol.h:119-129, hashPCG)
    sob_in = rng.integers(0, 1 << 32, (2048, 4), dtype=np.uint64).astype(np.uint32)
    sob_in[:256, 0] = np.arange(256)
    sob_out = np.zeros((2048, 2), np.float32)
    for i in range(2048):
        R.ref_sobol(*map(int, sob_in[i]), O.P(sob_out[i]))
    hp_in = rng.integers(0, 1 << 32, 2048, dtype=np.uint64).astype(np.uint32)
    hp_out = np.array([R.ref_hash_pcg(int(v)) for v in hp_in], np.uint32)
    np.savez_compressed(os.path.join(HERE, "samples.npz"), sobol_in=sob_in, sobol_out=sob_out, hash_in=hp_in,
                        hash_out=hp_out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
