#!/usr/bin/env python
"""AO Mrays/s and build Mtri/s of minimumlbvh_b200 on B200.

Workload (default ``soup4m_ao64``): a 4,194,304-triangle Gaussian-cluster soup
(64 clusters, sigma 0.02, lognormal edges), built into an LBVH, then one AO
frame at 1920 x 1080: one closest-hit primary ray per pixel and 64
Owen-Sobol cosine AO rays (radius 0.1) per hit. ``heightfield_ao16`` is the
212,992-triangle heightfield + icospheres scene at 512 x 512 with 16 AO rays
of radius 0.25.

A step is one AO frame (primary + AO rays) over the resident BVH; the build
is timed separately (one build per step) and reported in ``build``. ``e2e``
times the whole path through the C ABI from pinned HOST triangles: upload,
build, AO frame, download of the packed image.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload NAME]

Under torchrun (N > 1) every rank renders its own replica of the frame
(the path does not shard: the build is a global sort and a bottom-up climb,
and one frame's rays fit one GPU); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "soup4m_ao64": dict(scene="soup", n=4_194_304, w=1920, h=1080, ns=64, radius=0.1),
    "heightfield_ao16": dict(scene="heightfield", n=212_992, w=512, h=512, ns=16, radius=0.25),
}
METRIC = "AO Mrays/s (primary + AO rays, stack-free LBVH traversal)"
# algorithmic bytes per triangle of the build chain: 36 (bounds) + 36 (keys) + 8 (key write) + 8 (count)
# + 4 x 16 (four sort passes) + 9 (deltas) + 6 (index and delta reads) + 36 (leaf triangle) + 64 (node)
# + 24 (sibling box)
BUILD_BYTES_PER_TRI = 291


def make_scene(wl):
    from minimumlbvh_b200 import scenes
    if wl["scene"] == "soup":
        tris = scenes.gaussian_soup(wl["n"])
        cam = scenes.camera_soup()
    else:
        tris = scenes.heightfield_icospheres()
        cam = scenes.camera_heightfield()
    return tris, cam


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.lines = []
        self.device = device_index
        self.error = None

    def __enter__(self):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            ident = ["--id=GPU-" + uuid if not uuid.startswith("GPU-") else "--id=" + uuid]
        except Exception:
            ident = ["-i", str(self.device)]
        try:
            self.proc = subprocess.Popen(["nvidia-smi", *ident, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception as e:  # no nvidia-smi
            self.error = str(e)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                rows.append((float(p[0]), float(p[1]), p[4:8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "note": self.error or "no nvidia-smi samples"}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags) if f.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def onchip_peaks(dev, stream, reps: int = 10):
    """Bandwidths this project measures itself with its own probe kernel
    (mlbvh_read_probe: the traversal's 32-byte node load), CUDA events, best
    of `reps` launches after a warm-up: 32-byte sectors streamed and gathered
    at random from a 64 MiB buffer (resident in the 126 MB L2, beyond the
    L1s) and from a 4 GiB one (HBM). GB/s."""
    import torch
    import minimumlbvh_b200 as mb
    sink = torch.zeros(1024, dtype=torch.int32, device=dev)
    out = {}
    for where, nbytes in (("l2", 64 << 20), ("hbm", 4 << 30)):
        buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        buf.random_(0, 256)
        for pattern, name, loads in ((0, "stream", 64 if where == "l2" else 2), (1, "gather", 256)):
            best = 0.0
            for i in range(reps + 2):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                nread = mb.read_probe(buf, pattern, loads, sink, stream)
                b.record(stream)
                b.synchronize()
                if i >= 2:
                    best = max(best, nread / (a.elapsed_time(b) / 1e3) / 1e9)
            out[f"{where}_{name}_gbs"] = best
        del buf
    torch.cuda.synchronize()
    out["what"] = ("mlbvh_read_probe (ld.global.nc.v8, 32 B per load): 'stream' = consecutive sectors per warp, "
                   "'gather' = one random 32-byte sector per load; l2 = 64 MiB buffer, hbm = 4 GiB buffer; "
                   "best of 10 event-timed launches")
    out["launches"] = 4 * (reps + 2)
    return out


def committed_traffic(workload):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get(workload)


def cpu_sample_ao(wl, tris, cam_arr, out, seconds: float, rows=None):
    """Reference CPU AO (oracle/_ref: the reference's intersect_stackfree and
    sampling code, all host threads). With `rows` = (first, end) it times
    exactly those rows of the frame; else a band around the middle of the
    frame, grown until about `seconds` of wall time. Returns the baseline
    record, the elapsed seconds and the per-pixel occlusion counts (rows
    outside the band are 0)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O
    w, h = wl["w"], wl["h"]
    occ = np.zeros(w * h, np.uint32)
    nodes = out["nodes"]
    if O.ref_available():
        kind, L = "reference", O.ref()
        threads = L.ref_threads()

        def run(r0, r1):
            st = np.zeros(1, np.uint64)
            L.ref_ao_param(O.P(occ), w, h, O.P(cam_arr), out["root"], O.P(nodes), O.P(tris), wl["ns"],
                           float(wl["radius"]), 12345, r0, r1, O.P(st))
            return int(st[0])
    else:
        kind, L = "port", O.oracle()
        threads = int(os.environ.get("MLBVH_ORACLE_THREADS", os.cpu_count() or 1))

        def run(r0, r1):
            _, _, cnt = O.render_ao(cam_arr, out["root"], nodes, tris, w, h, wl["ns"], wl["radius"], 12345, 1,
                                    trig=0, rows=(r0, r1), counters=True)
            return int(cnt[2])
    if rows is not None:
        r0, r1 = rows
        t0 = time.perf_counter()
        rays = run(r0, r1)
        elapsed = time.perf_counter() - t0
    else:
        band, rays, elapsed = 2, 0, 0.0
        mid = h // 2
        while True:
            r0 = max(0, mid - band // 2)
            r1 = min(h, r0 + band)
            t0 = time.perf_counter()
            rays = run(r0, r1)
            elapsed = time.perf_counter() - t0
            if elapsed >= seconds or r1 - r0 >= h:
                break
            band = min(h, max(band * 2, int(band * seconds / max(elapsed, 1e-3))))
    return {"value": rays / elapsed / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
            "sample": f"AO rows {r0}-{r1 - 1} of the {w}x{h} frame ({rays} rays, {elapsed:.1f} s)"}, elapsed, occ


def cpu_rows(wl):
    """The rows both CPU legs (cpu_baseline and --impl reference) time: the
    whole frame, so that both run the same rays."""
    return (0, wl["h"])


def cpu_build_baseline(tris):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O
    n = len(tris)
    nodes = np.zeros((n - 1, 16), np.uint32)
    deltas = np.zeros(n - 1, np.uint8)
    root = np.zeros(1, np.uint32)
    if O.ref_available():
        t0 = time.perf_counter()
        O.ref().ref_cpu_builder(O.P(tris), n, 2, O.P(nodes), O.P(deltas), O.P(root))  # BVHCPUBuilder, parallel
        dt = time.perf_counter() - t0
        return {"mtri_s": n / dt / 1e6, "ms": dt * 1e3, "kind": "reference",
                "what": "BVHCPUBuilder::build with BUILD_OPTION_CPU_PARALLEL"}
    t0 = time.perf_counter()
    O.build(tris)
    dt = time.perf_counter() - t0
    return {"mtri_s": n / dt / 1e6, "ms": dt * 1e3, "kind": "port", "what": "oracle build (serial)"}


def oracle_agreement(wl, tris, cam_arr, out, occ_plain, form_occ, occ_ref, ref_kind):
    """Per-pixel occlusion counts of the timed frame (plain form and every
    other form) against the oracle's restatement over the whole frame, with
    this project's FP32 sincos for the sample directions as the kernels use
    it (all host threads; outside the timed regions), and the plain form
    against the reference's own CPU code (its libm sincos: a few AO rays
    differ by an ulp of direction)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O
    w, h = wl["w"], wl["h"]
    t0 = time.perf_counter()
    _, occ_oracle = O.render_ao(cam_arr, out["root"], out["nodes"], tris, w, h, wl["ns"], wl["radius"], 12345, 1,
                                trig=1)
    res = {"pixels": int(w * h), "oracle_s": time.perf_counter() - t0,
           "plain": float((occ_plain == occ_oracle).mean())}
    for name, occ in form_occ.items():
        res[name] = float((occ == occ_oracle).mean())
    res["plain_vs_reference_cpu"] = float((occ_plain == occ_ref).mean())
    res["reference_cpu_kind"] = ref_kind
    return res


def bench_batched(args, dev, stream, barrier, max_over_ranks, world, n_meshes=1024, autotune=True):
    """The batched workload: 1,024 meshes with log-uniform 64..262,144
    triangles (30.8M in all) and log-uniform 4,096..1,048,576 incoherent rays
    each (169M), generated on the device. Build + traversal run as one CUDA
    graph launch with autotuned parameters; the plain form is the same work as
    1,024 mlbvh_build + 1,024 mlbvh_trace calls. Inputs are larger than L2."""
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import scenes
    tris, offsets = scenes.batched_soup(n_meshes, 64, 262_144, seed=7, device=dev)
    rays, roff = scenes.batched_rays(tris, offsets, 4096, 1_048_576, seed=8)
    nm, n, nr = len(offsets) - 1, int(offsets[-1]), int(roff[-1])
    bb = mb.BatchedBVH(tris, torch.as_tensor(offsets.astype(np.int32), device=dev), nm)
    bb.set_rays(rays, torch.as_tensor(roff.astype(np.int32), device=dev))
    if autotune:
        params, tune_build_ms, tune_trace_ms = bb.autotune()
    else:
        params, tune_build_ms, tune_trace_ms = mb.BatchParams.default(), None, None
        bb.build(params)
    bb.status()
    graph = bb.graph(params, stages=3)
    steps = max(1, args.steps)
    for _ in range(args.warmup):
        graph.launch()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    bev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    tev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    for i in range(steps):
        ev[i][0].record(stream)
        graph.launch()
        ev[i][1].record(stream)
    for i in range(steps):
        bev[i][0].record(stream)
        mb.profile_events(*kev[i])  # around k_batch_build, the climb
        bb.build(params)
        bev[i][1].record(stream)
        tev[i][0].record(stream)
        bb.trace(params)
        tev[i][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    bb.status()
    graph.close()
    graph_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3 / steps)
    build_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in bev) / 1e3 / steps)
    trace_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in tev) / 1e3 / steps)
    climb_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in kev) / 1e3 / steps)
    hits = bb.hits.clone()

    # the plain form: the same meshes and rays, one mesh per call
    meshes = [tris[int(offsets[m]):int(offsets[m + 1])].clone() for m in range(nm)]
    builders = [mb.BVHGPUBuilder() for _ in range(nm)]
    sorter = mb.OnesweepSort(dev.index)
    sorter.reserve(mb.lib().mlbvh_build_scratch_bytes(int(np.diff(offsets).max())))
    plain_hits = torch.empty_like(hits)

    def plain_build():
        for m in range(nm):
            builders[m].build(meshes[m], meshes[m].shape[0], 0, sorter)

    def plain_trace():
        for m in range(nm):
            r0, r1 = int(roff[m]), int(roff[m + 1])
            mb.intersect(builders[m], meshes[m], rays[r0:r1], hits=plain_hits[r0:r1])

    plain_build()
    plain_trace()
    torch.cuda.synchronize()
    pev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    barrier()
    torch.cuda.synchronize()
    pev[0].record(stream)
    plain_build()
    pev[1].record(stream)
    plain_trace()
    pev[2].record(stream)
    torch.cuda.synchronize()
    barrier()
    pb_s = max_over_ranks(pev[0].elapsed_time(pev[1]) / 1e3)
    pt_s = max_over_ranks(pev[1].elapsed_time(pev[2]) / 1e3)
    agree = float((plain_hits == hits).all(1).double().mean().item())
    return {
        "workload": f"batched{nm}", "meshes": nm, "triangles": n, "rays": nr,
        "value": nr * world / trace_s / 1e6, "unit": "Mrays/s (persistent queue traversal)",
        "build_ms": build_s * 1e3, "climb_ms": climb_s * 1e3, "build_mtri_s": n * world / build_s / 1e6,
        "trace_ms": trace_s * 1e3,
        "graph_ms": graph_s * 1e3, "graph_mrays_s": nr * world / graph_s / 1e6,
        "plain_build_ms": pb_s * 1e3, "plain_trace_ms": pt_s * 1e3, "plain_mrays_s": nr * world / pt_s / 1e6,
        "vs_plain_trace": pt_s / trace_s, "vs_plain_build": pb_s / build_s,
        "vs_plain_build_plus_trace": (pb_s + pt_s) / graph_s, "hit_agreement": agree,
        "params": params.as_dict(), "autotune_ms": {"build": tune_build_ms, "trace": tune_trace_ms},
        # graph (8 build kernels + traversal) and direct build + traversal per step; the plain loop once
        "launches": steps * 18 + 8 * nm,
    }


def bench_precision(args, builder, qtree, wide, d_tris, tris, cam, w, h, dev, stream, max_over_ranks):
    """The precision configuration: closest hits of 1M camera rays of the
    frame (every other pixel) over the FP32 and the quantised trees, each at
    the same walk: the binary tree's replay walk (64-byte nodes against the
    quantised 32-byte nodes) and the 4-wide tree's closest-hit walk (128-byte
    slots against 64-byte quantised slots), beside the plain form (the
    reference's stack-free walk). Hit-ID agreement and t equality with the
    plain form, the largest t error against the FP64 evaluation of the
    ray-plane formula (with its stated bound, fp64check), node bytes per ray,
    and Mrays/s (rays resident, CUDA events)."""
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import fp64check, scenes
    rays_h = scenes.camera_rays(cam.m_origin, cam.m_right, cam.m_up, w, h, 2)
    n = len(rays_h)
    rays = torch.from_numpy(rays_h).to(dev)
    closest = mb.RAY_QUERY_CLOSEST

    def run(fn):
        for _ in range(args.warmup):
            fn()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(ev[0].elapsed_time(ev[1]) / 1e3 / args.steps)

    hits = {k: torch.empty((n, 8), dtype=torch.int32, device=dev) for k in
            ("plain", "replay", "quantised_replay", "wide", "wide_quantised")}
    calls = {
        "plain": lambda: mb.intersect(builder, d_tris, rays, hits=hits["plain"]),
        "replay": lambda: mb.intersect(builder, d_tris, rays, traversal=mb.TRAVERSAL_REPLAY, hits=hits["replay"]),
        "quantised_replay": lambda: mb.intersect_quantised(qtree, rays, closest, hits=hits["quantised_replay"]),
        "wide": lambda: mb.intersect_wide(wide, rays, hits=hits["wide"], rayQuery=closest),
        "wide_quantised": lambda: mb.intersect_wide(wide, rays, hits=hits["wide_quantised"], quantised=True,
                                                    rayQuery=closest),
    }
    # node bytes per ray from the counting variants
    cq = torch.zeros(3 * n, dtype=torch.int32, device=dev)
    mb.intersect_quantised(qtree, rays, closest, stack_depth=16, counts=cq)
    cw = torch.zeros(3 * n, dtype=torch.int32, device=dev)
    mb.intersect_wide(wide, rays, counts=cw, rayQuery=closest)
    cwq = torch.zeros(3 * n, dtype=torch.int32, device=dev)
    mb.intersect_wide(wide, rays, counts=cwq, quantised=True, rayQuery=closest)
    times = {k: run(f) for k, f in calls.items()}
    host = {k: v.cpu().numpy().view(np.uint32) for k, v in hits.items()}
    c = cq.cpu().numpy().astype(np.int64)
    cwh = cw.cpu().numpy().astype(np.int64)
    cwqh = cwq.cpu().numpy().astype(np.int64)
    a = host["plain"]
    forms = {}
    node_bytes = {"quantised_replay": (32 * c[:n].sum() + 4 * c[2 * n:].sum()) / n,
                  "wide": 128 * cwh[:n].sum() / n, "wide_quantised": 64 * cwqh[:n].sum() / n}
    for k in calls:
        b = host[k]
        forms[k] = {"mrays_s": n / times[k] / 1e6, "vs_plain": times["plain"] / times[k],
                    "hit_id_agreement": float((a[:, 7] == b[:, 7]).mean()),
                    "t_equal": float((a[:, 0] == b[:, 0]).mean())}
        if k in node_bytes:
            forms[k]["node_bytes_per_ray"] = node_bytes[k]
    chk = fp64check.check_hits(tris, rays_h, host["quantised_replay"])
    chkw = fp64check.check_hits(tris, rays_h, host["wide_quantised"])
    return {
        "rays": n, "rays_desc": f"camera rays of every other pixel of the {w}x{h} frame, closest hit",
        "hit_id_agreement": forms["quantised_replay"]["hit_id_agreement"],
        "t_equal": forms["quantised_replay"]["t_equal"],
        "hits": chk["hits"], "max_abs_t_err_vs_fp64": chk["max_abs_err"], "max_rel_t_err_vs_fp64": chk["max_rel_err"],
        "max_t_err_over_bound": chk["max_bound_ratio"],
        "wide_quantised_max_t_err_over_bound": chkw["max_bound_ratio"],
        "node_bytes_per_ray": node_bytes["quantised_replay"],
        "quantised_mrays_s": forms["quantised_replay"]["mrays_s"], "plain_mrays_s": forms["plain"]["mrays_s"],
        "vs_plain": forms["quantised_replay"]["vs_plain"],
        "equal_walk": {"quantised_vs_fp32_binary_replay": times["replay"] / times["quantised_replay"],
                       "quantised_vs_fp32_wide": times["wide"] / times["wide_quantised"]},
        "best": max(forms, key=lambda k: forms[k]["mrays_s"] if forms[k]["hit_id_agreement"] == 1.0 else 0),
        "forms": forms,
        "launches": 3 + (len(calls)) * (args.warmup + args.steps),
    }


def bench_precision_heightfield(args, dev, stream, max_over_ranks):
    """The precision configuration on the other scene: the heightfield +
    icospheres (212,992 triangles), camera rays of every other pixel of a
    1448x1448 frame (1,048,352 rays, the same count as the soup's), the same
    forms and checks as bench_precision."""
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import scenes
    tris = scenes.heightfield_icospheres()
    n = len(tris)
    d_tris = torch.from_numpy(tris).to(dev)
    builder = mb.BVHGPUBuilder().build(d_tris, n, 0, mb.OnesweepSort(dev.index))
    builder.status()
    qtree = mb.QuantisedBVH.from_builder(builder, d_tris)
    wide = mb.WideBVH.from_builder(builder, d_tris).quantise()
    w = h = 1448
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
    out = bench_precision(args, builder, qtree, wide, d_tris, tris, cam, w, h, dev, stream, max_over_ranks)
    out["workload"] = f"heightfield + icospheres ({n:,} triangles)"
    return out


def bench_pt(args, dev, stream, max_over_ranks, reference_gpu=False):
    """Path tracing (pt, main_gpu.cu:179-272) on the 212,992-triangle
    heightfield + icospheres scene with 1 % emissive triangles, 512 x 512,
    Owen-Sobol samples, the reference's 1024-bounce limit with Russian
    roulette: progressive passes (one sample per pixel each) with the
    stack-free walk and with the replay walk over leaf-ordered triangles,
    which must leave bit-identical accumulators. With ``reference_gpu`` (one
    process only) the reference's own pt kernel, compiled unmodified for
    sm_100a (oracle/_ref/libmlbvh_ref_gpu.so), runs the same passes over the
    same tree for comparison."""
    import ctypes
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import scenes
    tris = scenes.heightfield_icospheres()
    n = len(tris)
    t = torch.from_numpy(tris).to(dev)
    at = torch.from_numpy(scenes.pt_attributes(n, light_fraction=0.01)).to(dev)
    b = mb.BVHGPUBuilder().build(t, n, 0, mb.OnesweepSort(dev.index))
    b.status()
    lt = mb.leaf_triangles(b, t)
    eye, c, up, fovy = scenes.camera_heightfield()
    w = h = 512
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
    out = {}
    accs = {}
    for name, kw in (("plain", {}), ("replay", {"traversal": mb.TRAVERSAL_REPLAY, "leaf_triangles": lt})):
        acc = torch.zeros((w * h, 4), dtype=torch.float32, device=dev)
        for _ in range(args.warmup):
            mb.render_pt(acc, (w, h), cam, b.m_rootNode, b.m_internals, t, at, 1, **kw)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            mb.render_pt(acc, (w, h), cam, b.m_rootNode, b.m_internals, t, at, 1, **kw)
        ev[1].record(stream)
        torch.cuda.synchronize()
        sec = max_over_ranks(ev[0].elapsed_time(ev[1]) / 1e3)
        out[name] = {"ms_per_pass": sec * 1e3 / args.steps, "msamples_s": w * h * args.steps / sec / 1e6}
        accs[name] = acc
    out["replay"]["vs_plain"] = out["plain"]["ms_per_pass"] / out["replay"]["ms_per_pass"]
    out["replay"]["accumulators_equal"] = bool(torch.equal(accs["plain"], accs["replay"]))
    if not args.no_ploc:
        # the replay walk over the higher-quality (PLOC, radius 8) tree of the same
        # triangles: the same closest distances; a path may take another branch
        # only where two triangles meet a ray at the same distance
        pb = mb.BVHGPUBuilder().buildByPLOC(t, n, 0, mb.OnesweepSort(dev.index), 8)
        pb.status()
        plt = mb.leaf_triangles(pb, t)
        acc = torch.zeros((w * h, 4), dtype=torch.float32, device=dev)
        for _ in range(args.warmup):
            mb.render_pt(acc, (w, h), cam, pb.m_rootNode, pb.m_internals, t, at, 1, traversal=mb.TRAVERSAL_REPLAY,
                         leaf_triangles=plt)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            mb.render_pt(acc, (w, h), cam, pb.m_rootNode, pb.m_internals, t, at, 1, traversal=mb.TRAVERSAL_REPLAY,
                         leaf_triangles=plt)
        ev[1].record(stream)
        torch.cuda.synchronize()
        sec = max_over_ranks(ev[0].elapsed_time(ev[1]) / 1e3)

        def mean_rad(a):
            a = a.double()
            return float(a[:, :3].sum() / a[:, 3].sum())
        out["ploc_replay"] = {"ms_per_pass": sec * 1e3 / args.steps, "msamples_s": w * h * args.steps / sec / 1e6,
                              "vs_lbvh_replay": out["replay"]["ms_per_pass"] / (sec * 1e3 / args.steps),
                              "vs_plain": out["plain"]["ms_per_pass"] / (sec * 1e3 / args.steps),
                              "mean_radiance": mean_rad(acc), "lbvh_mean_radiance": mean_rad(accs["replay"]),
                              "pixels_equal_to_lbvh": float((acc == accs["replay"]).all(1).double().mean().item())}
    out["workload"] = "heightfield + icospheres (212,992 triangles), 512x512, 1 % emissive, up to 1024 bounces"
    if reference_gpu and os.path.exists(REF_GPU_LIB):
        # 512 is a multiple of the reference's 16 x 16 blocks: its grid covers the image exactly
        L = ctypes.CDLL(REF_GPU_LIB)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.refgpu_pt.argtypes = [vp, i64, i32, i32, vp, vp, vp, vp, vp, i32, i32, vp]
        L.refgpu_pt.restype = i32
        cam_arr = np.ascontiguousarray(cam.as_array(), np.float32)
        acc = torch.zeros((w * h, 4), dtype=torch.float32, device=dev)

        def ref_pass():
            rc = L.refgpu_pt(mb._ptr(acc), w * h, w, h, cam_arr.ctypes.data, mb._ptr(b.m_rootNode),
                             mb._ptr(b.m_internals), mb._ptr(t), mb._ptr(at), 1, 1 << 30, stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(f"reference GPU pt: status {rc}")
        for _ in range(args.warmup):
            ref_pass()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            ref_pass()
        ev[1].record(stream)
        torch.cuda.synchronize()
        sec = ev[0].elapsed_time(ev[1]) / 1e3

        def mean_radiance(a):
            a = a.double()
            return float(a[:, :3].sum() / a[:, 3].sum())
        ref_mean, our_mean = mean_radiance(acc), mean_radiance(accs["plain"])
        out["reference_gpu"] = {
            "what": "the reference's own pt kernel (main_gpu.cu) compiled unmodified for sm_100a, 16x16 blocks, "
                    "over the same tree and inputs",
            "ms_per_pass": sec * 1e3 / args.steps, "msamples_s": w * h * args.steps / sec / 1e6,
            "plain_vs_reference": sec / args.steps / (out["plain"]["ms_per_pass"] / 1e3),
            "replay_vs_reference": sec / args.steps / (out["replay"]["ms_per_pass"] / 1e3),
            "mean_radiance_reference": ref_mean, "mean_radiance_ours": our_mean,
            "accumulators_equal": bool(torch.equal(acc, accs["plain"])),
            "note": "the reference is compiled with nvcc's default FMA contraction and CUDA's cosf/sinf; ours "
                    "rounds like the reference's host code, so individual paths may diverge while the image "
                    "means agree",
        }
    return out


def bench_diff(args, dev, stream, max_over_ranks):
    """Differentiable path tracing and its path-replay adjoint on the
    heightfield + icospheres scene with a 0.5 x 0.5 quad light of radiance 10
    (212,994 triangles), per-triangle grey albedo uniform in [0.1, 0.9], 512 x
    512 at 64 samples per pixel, 3 bounces: the forward render, the L2 loss
    against a target rendered with a second albedo seed, and the adjoint
    giving dLoss/dAlbedo for every triangle (paths recomputed from their
    seeds). Timed with CUDA events. A directional finite difference of the
    loss (GPU renders at albedo +- eps along a random direction over the
    triangles with the largest gradients) against the gradient's projection
    checks the adjoint without the host oracle."""
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import scenes
    tris, alb, em = scenes.diff_scene()
    n = len(tris)
    t = torch.from_numpy(tris).to(dev)
    b = mb.BVHGPUBuilder().build(t, n, 0, mb.OnesweepSort(dev.index))
    b.status()
    w = h = 512
    spp, bounces = 64, 3
    eye, c, up, fovy = scenes.camera_heightfield()
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
    a = torch.from_numpy(alb).to(dev)
    e = torch.from_numpy(em).to(dev)
    target = torch.empty(w * h, dtype=torch.float32, device=dev)
    mb.pt_diff_render(target, (w, h), cam, b, t, torch.from_numpy(scenes.albedo(n, 2)).to(dev), e, spp, bounces)
    img = torch.empty_like(target)
    grad = torch.zeros(n, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(ev[0].elapsed_time(ev[1]) / 1e3) / args.steps

    t_fwd = timed(lambda: mb.pt_diff_render(img, (w, h), cam, b, t, a, e, spp, bounces))
    gimg = 2.0 * (img - target)

    def adjoint():
        grad.zero_()
        mb.pt_diff_adjoint(grad, gimg, (w, h), cam, b, t, a, e, spp, bounces)
    t_adj = timed(adjoint)

    def loss(albedo):
        mb.pt_diff_render(img, (w, h), cam, b, t, albedo, e, spp, bounces)
        return float(((img.double() - target.double()) ** 2).sum().item())
    g = grad.double()
    top = torch.topk(g.abs(), 1000).indices
    rng = torch.Generator(device="cpu").manual_seed(11)
    v = torch.zeros(n, dtype=torch.float64, device=dev)
    v[top] = (torch.rand(1000, generator=rng, dtype=torch.float64) * 2 - 1).to(dev)
    eps = 1e-2
    fd = (loss((a.double() + eps * v).float()) - loss((a.double() - eps * v).float())) / (2 * eps)
    proj = float((g * v).sum().item())
    paths = w * h * spp
    return {"workload": "heightfield + icospheres + quad light (212,994 triangles), 512x512, 64 spp, 3 bounces",
            "forward_ms": t_fwd * 1e3, "forward_mpaths_s": paths / t_fwd / 1e6,
            "adjoint_ms": t_adj * 1e3, "adjoint_mpaths_s": paths / t_adj / 1e6,
            "adjoint_vs_forward": t_adj / t_fwd,
            "directional_check": {"finite_difference": fd, "gradient_projection": proj,
                                  "rel_err": abs(fd - proj) / max(abs(proj), 1e-30), "eps": eps,
                                  "direction": "random in [-1, 1] on the 1,000 triangles with the largest gradients"},
            "launches": 2 * (args.warmup + args.steps) + 10}  # + target and two FD renders, 7 build launches


def sah_cost_device(nodes, root_t):
    """Surface-area cost of a tree on the device: half areas of every internal
    node's box and of every leaf's box over the root box's (unit costs)."""
    import torch
    nd = nodes
    box = nd[:, 2:14].view(torch.float32).double().reshape(-1, 2, 6)
    lo = torch.minimum(box[:, 0, :3], box[:, 1, :3])
    hi = torch.maximum(box[:, 0, 3:], box[:, 1, 3:])

    def half(l, h):
        d = h - l
        return d[..., 0] * d[..., 1] + d[..., 1] * d[..., 2] + d[..., 2] * d[..., 0]
    leaf = nd[:, :2] < 0  # leaf bit (bit 31)
    total = half(lo, hi).sum() + (half(box[..., :3], box[..., 3:]) * leaf).sum()
    r = int(root_t[0].item())
    return float(total / half(lo[r], hi[r]))


def bench_ploc(args, wl, d_tris, n, cam, w, h, dev, stream, barrier, max_over_ranks, flush, lbvh, lbvh_forms,
               occ_plain):
    """The higher-quality build (mlbvh_build_ploc, radius 8; the reference's
    counterpart is Embree's SAH build behind buildByEmbree, which cannot run
    here) on the same scene: build time against the LBVH's, surface-area
    cost of both trees, and AO frames over the PLOC tree (plain stack-free,
    replay and 4-wide forms) against the same forms over the LBVH, with the
    occlusion counts of every pixel compared with the LBVH's plain frame."""
    import torch
    import minimumlbvh_b200 as mb
    launches = 0
    pb = mb.BVHGPUBuilder()
    ps = mb.OnesweepSort(dev.index)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    bev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for _ in range(args.warmup):
        pb.buildByPLOC(d_tris, n, 0, ps, 8)
    pb.status()
    barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        if flush is not None:
            flush.zero_()
        bev[i][0].record(stream)
        mb.profile_events(*kev[i])
        pb.buildByPLOC(d_tris, n, 0, ps, 8)
        bev[i][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    pb.status()
    launches += 8 * (args.warmup + args.steps)  # bounds, keys, 4 sort passes, init, the cooperative k_ploc
    build_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in bev) / 1e3) / args.steps
    kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in kev]))
    sah_ploc = sah_cost_device(pb.m_internals[: n - 1], pb.m_rootNode)
    sah_lbvh = sah_cost_device(lbvh.m_internals[: n - 1], lbvh.m_rootNode)

    lt = mb.leaf_triangles(pb, d_tris)
    wide = mb.WideBVH.from_builder(pb, d_tris)
    launches += 3
    px = torch.zeros(w * h, dtype=torch.int32, device=dev)

    def plain(occluded=None):
        mb.render_ao(px, (w, h), cam, pb.m_rootNode, pb.m_internals, d_tris, 1, wl["ns"], wl["radius"], 12345,
                     occluded=occluded)

    def replay(occluded=None):
        mb.render_ao(px, (w, h), cam, pb.m_rootNode, pb.m_internals, d_tris, 1, wl["ns"], wl["radius"], 12345,
                     occluded=occluded, traversal=mb.TRAVERSAL_REPLAY, leaf_triangles=lt)

    def wide_form(occluded=None):
        mb.render_ao_wide(px, (w, h), cam, wide, 1, wl["ns"], wl["radius"], 12345, occluded=occluded)

    out = {"radius": 8, "build_ms": build_s * 1e3, "build_mtri_s": n / build_s / 1e6,
           "k_ploc_ms": kernel_ms, "lbvh_build_ms": lbvh_forms["build_ms"],
           "sah_cost": sah_ploc, "lbvh_sah_cost": sah_lbvh, "sah_vs_lbvh": sah_ploc / sah_lbvh, "forms": {}}
    for name, frame in (("plain", plain), ("replay", replay), ("wide", wide_form)):
        occ = torch.empty_like(occ_plain)
        frame(occluded=occ)
        for _ in range(args.warmup):
            frame()
        fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            if flush is not None:
                flush.zero_()
            fev[i][0].record(stream)
            frame()
            fev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        launches += 3 * (1 + args.warmup + args.steps)
        t = max_over_ranks(sum(a.elapsed_time(b) for a, b in fev) / 1e3) / args.steps
        lb_ms = lbvh_forms[name]
        out["forms"][name] = {"ms_per_frame": t * 1e3, "mrays_s": lbvh_forms["rays_per_frame"] / t / 1e6,
                              "lbvh_ms_per_frame": lb_ms, "vs_lbvh_same_form": lb_ms / (t * 1e3),
                              "occlusion_agreement_with_lbvh": float((occ == occ_plain).double().mean().item())}
    # closest hits of camera rays (every other pixel of the frame): the replay
    # walk over both trees; the same distances (the triangle may differ only
    # where two meet a ray at the same distance)
    from minimumlbvh_b200 import scenes
    rays = torch.from_numpy(scenes.camera_rays(cam.m_origin, cam.m_right, cam.m_up, w, h, 2)).to(dev)
    nr = rays.shape[0]
    hits = {}
    cam_out = {"rays": nr}
    for name, bld in (("lbvh", lbvh), ("ploc", pb)):
        hb = torch.empty((nr, 8), dtype=torch.int32, device=dev)
        for _ in range(args.warmup):
            mb.intersect(bld, d_tris, rays, traversal=mb.TRAVERSAL_REPLAY, hits=hb)
        cev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        cev[0].record(stream)
        for _ in range(args.steps):
            mb.intersect(bld, d_tris, rays, traversal=mb.TRAVERSAL_REPLAY, hits=hb)
        cev[1].record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(cev[0].elapsed_time(cev[1]) / 1e3) / args.steps
        launches += args.warmup + args.steps
        cam_out[name + "_mrays_s"] = nr / t / 1e6
        hits[name] = hb
    cam_out["vs_lbvh"] = cam_out["ploc_mrays_s"] / cam_out["lbvh_mrays_s"]
    cam_out["t_equal"] = float((hits["lbvh"][:, 0] == hits["ploc"][:, 0]).double().mean().item())
    cam_out["triangle_equal"] = float((hits["lbvh"][:, 7] == hits["ploc"][:, 7]).double().mean().item())
    # the same rays on the closest-hit walk over each tree's 4-wide regrouping
    # (leaf-ordered triangles: neighbouring leaves share cache lines), with
    # the walk's per-ray wide-node visits and triangle tests
    lbvh_wide = mb.WideBVH.from_builder(lbvh, d_tris)
    launches += 2
    for name, wt in (("lbvh", lbvh_wide), ("ploc", wide)):
        hw = torch.empty((nr, 8), dtype=torch.int32, device=dev)
        cnt = torch.zeros(3 * nr, dtype=torch.int32, device=dev)
        mb.intersect_wide(wt, rays, hits=hw, counts=cnt, rayQuery=mb.RAY_QUERY_CLOSEST)
        for _ in range(args.warmup):
            mb.intersect_wide(wt, rays, hits=hw, rayQuery=mb.RAY_QUERY_CLOSEST)
        cev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        cev[0].record(stream)
        for _ in range(args.steps):
            mb.intersect_wide(wt, rays, hits=hw, rayQuery=mb.RAY_QUERY_CLOSEST)
        cev[1].record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(cev[0].elapsed_time(cev[1]) / 1e3) / args.steps
        launches += 1 + args.warmup + args.steps
        c = cnt.cpu().numpy().astype(np.int64)
        cam_out[name + "_wide_mrays_s"] = nr / t / 1e6
        cam_out[name + "_wide_node_visits_per_ray"] = c[:nr].sum() / nr
        cam_out[name + "_wide_tri_tests_per_ray"] = c[nr:2 * nr].sum() / nr
        cam_out[name + "_wide_t_equal_replay"] = float((hw[:, 0] == hits[name][:, 0]).double().mean().item())
    cam_out["wide_vs_lbvh"] = cam_out["ploc_wide_mrays_s"] / cam_out["lbvh_wide_mrays_s"]
    out["camera_rays_closest"] = cam_out
    out["launches"] = launches
    out["note"] = ("PLOC: parallel locally-ordered clustering over the LBVH's Morton order, in-order node numbering "
                   "(the LBVH's conventions), one cooperative kernel after the shared key and sort passes")
    return out


REF_GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libmlbvh_ref_gpu.so")


def bench_reference_gpu(args, builder, sorter, d_tris, n, cam, w, h, dev, stream, max_over_ranks):
    """Baseline leg: the reference's OWN GPU kernels, compiled unmodified for
    sm_100a (oracle/_ref/libmlbvh_ref_gpu.so, built from the reference sources
    by oracle/Makefile), against this project's kernels on the same B200.

    Build: the reference's getSceneAABB + buildMortons, and computeDeltas +
    0xFF fill + build over sorted pairs. Its Onesweep sort is not run (its waits
    are unbounded; see oracle/ref_gpu_launch.cu): the pairs come from this
    project's sort, which produces the reference's stable order, so the sort is
    excluded from the reference's time and included in ours. AO: the
    reference's ao kernel, which fixes 16 Owen-Sobol samples of length 1.0
    (main_gpu.cu:148, 165), over the validated tree, against the plain and the
    4-wide forms at the same 16 samples and radius 1.0. The reference's grid
    also covers the rows up to the next multiple of 16 (a padded buffer takes
    its writes); only the frame's rays are counted."""
    import ctypes
    import torch
    import minimumlbvh_b200 as mb
    if not os.path.exists(REF_GPU_LIB):
        return {"unavailable": "oracle/_ref/libmlbvh_ref_gpu.so is not built (it needs the reference sources)"}
    L = ctypes.CDLL(REF_GPU_LIB)
    vp, i32, i64, u32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_uint32
    L.refgpu_scene_aabb.argtypes = [vp, vp, i32, vp]
    L.refgpu_mortons.argtypes = [vp, vp, i32, vp, u32, vp]
    L.refgpu_deltas_and_build.argtypes = [vp, vp, vp, i32, vp, vp, vp]
    L.refgpu_ao.argtypes = [vp, i64, i32, i32, vp, vp, vp, vp, i32, vp]
    for f in (L.refgpu_scene_aabb, L.refgpu_mortons, L.refgpu_deltas_and_build, L.refgpu_ao):
        f.restype = i32
    if (n - 1) % 256 == 0:
        return {"unavailable": "n - 1 is a multiple of 256: the reference's build grid would skip a leaf"}
    sp = stream.cuda_stream
    ptr = mb._ptr

    def check(rc, what):
        if rc != 0:
            raise RuntimeError(f"reference GPU {what}: status {rc}")

    # our build with the sorted pairs kept: the reference's input to computeDeltas + build
    builder.build(d_tris, n, 0, sorter, keep_keys=True)
    builder.status()
    pairs = torch.stack([builder.m_sortedKeys, builder.m_sortedIndices], 1).contiguous()
    scene = torch.empty(8, dtype=torch.float32, device=dev)
    mortons = torch.empty((n, 2), dtype=torch.int32, device=dev)
    deltas = torch.empty(n, dtype=torch.uint8, device=dev)
    nodes = torch.empty((n - 1, 16), dtype=torch.int32, device=dev)
    root = torch.empty(4, dtype=torch.int32, device=dev)

    def ref_build():
        check(L.refgpu_scene_aabb(ptr(scene), ptr(d_tris), n, sp), "getSceneAABB")
        check(L.refgpu_mortons(ptr(mortons), ptr(d_tris), n, ptr(scene), 0, sp), "buildMortons")
        check(L.refgpu_deltas_and_build(ptr(root), ptr(nodes), ptr(d_tris), n, ptr(deltas), ptr(pairs), sp),
              "computeDeltas/build")

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in ev])) / 1e3)

    ref_build_s = timed(ref_build, args.steps)
    ours_build_s = timed(lambda: builder.build(d_tris, n, 0, sorter), args.steps)
    # the reference's keys (unsorted, from its buildMortons) sorted stably must be ours
    ref_keys = mortons[:, 0].cpu().numpy().view(np.uint32)
    our_keys = pairs[:, 0].cpu().numpy().view(np.uint32)
    keys_equal = bool((np.sort(ref_keys, kind="stable") == our_keys).all())
    tree_equal = bool(torch.equal(nodes, builder.m_internals[: n - 1]) and torch.equal(root[:1], builder.m_rootNode[:1]))

    # AO at the reference's fixed parameters, over this project's tree (the
    # reference's own only if identical): 16 samples, length 1.0
    pw, ph = -(-w // 16) * 16, -(-h // 16) * 16
    ref_px = torch.zeros(pw * ph, dtype=torch.int32, device=dev)
    cam_arr = np.ascontiguousarray(cam.as_array(), np.float32)
    src_nodes = nodes if tree_equal else builder.m_internals
    src_root = root if tree_equal else builder.m_rootNode
    ref_ao_s = timed(lambda: check(L.refgpu_ao(ptr(ref_px), pw * ph, w, h, cam_arr.ctypes.data, ptr(src_root),
                                              ptr(src_nodes), ptr(d_tris), 1, sp), "ao"), args.steps)
    px = torch.zeros(w * h, dtype=torch.int32, device=dev)
    occ = torch.zeros(w * h, dtype=torch.int32, device=dev)
    plain_s = timed(lambda: mb.render_ao(px, (w, h), cam, builder.m_rootNode, builder.m_internals, d_tris, 1, 16, 1.0,
                                         12345, occluded=occ), args.steps)
    plain_px = px.clone()
    wide = mb.WideBVH.from_builder(builder, d_tris)
    wide_s = timed(lambda: mb.render_ao_wide(px, (w, h), cam, wide, 1, 16, 1.0, 12345), args.steps)
    torch.cuda.synchronize()
    rays = w * h + 16 * int((occ != -1).sum().item())
    a = ref_px.cpu().numpy().view(np.uint32)[: w * h]
    b = plain_px.cpu().numpy().view(np.uint32)
    ch = np.abs(np.stack([(a >> k) & 255 for k in (0, 8, 16)], 1).astype(np.int32)
                - np.stack([(b >> k) & 255 for k in (0, 8, 16)], 1).astype(np.int32)).max(1)
    return {
        "what": "the reference's own CUDA kernels (minimum_lbvh.cu, main_gpu.cu) compiled unmodified for sm_100a "
                "and launched with its own grids, on the same B200 and inputs",
        "build": {"reference_ms": ref_build_s * 1e3, "ours_ms": ours_build_s * 1e3,
                  "vs_reference": ref_build_s / ours_build_s, "reference_tree_equal": tree_equal,
                  "reference_keys_equal": keys_equal,
                  "note": "reference time excludes its Onesweep sort (not run: unbounded waits); ours includes our "
                          "sort"},
        "ao": {"samples": 16, "radius": 1.0, "rays_per_frame": rays,
               "reference_ms": ref_ao_s * 1e3, "reference_mrays_s": rays / ref_ao_s / 1e6,
               "plain_ms": plain_s * 1e3, "plain_mrays_s": rays / plain_s / 1e6, "plain_vs_reference": ref_ao_s / plain_s,
               "wide_ms": wide_s * 1e3, "wide_mrays_s": rays / wide_s / 1e6, "wide_vs_reference": ref_ao_s / wide_s,
               "pixels_equal": float((ch == 0).mean()), "max_channel_diff": int(ch.max()),
               "note": "the reference samples directions with CUDA's cosf/sinf, the plain form with its own FP32 "
                       "sincos: a few AO rays flip; the reference's grid also traces the padding rows "
                       f"{h}..{ph - 1} (uncounted)"},
    }


def run_reference(args, wl, rank):
    """The reference's own CPU implementation of the path, all host threads."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O
    tris, (eye, c, up, fovy) = make_scene(wl)
    out = O.build(tris)
    cam_arr = O.lookat(eye, c, up, fovy, wl["w"], wl["h"])
    values = []
    sample = None
    for i in range(args.warmup + args.steps):
        # the whole frame, the same rays as the cpu_baseline leg of this bench's own arm
        s, _, _ = cpu_sample_ao(wl, tris, cam_arr, out, seconds=args.ref_seconds, rows=cpu_rows(wl))
        if i >= args.warmup:
            values.append(s["value"])
            sample = s
    value = float(np.median(values))
    build = cpu_build_baseline(tris)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "triangles": wl["n"], "image": [wl["w"], wl["h"]],
                   "ao_samples": wl["ns"], "ao_radius": wl["radius"], "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": sample["cores"], "kind": sample["kind"],
                         "sample": sample["sample"]},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "build": build,
    }
    print(json.dumps(line), flush=True)


PROFILE_CASES = ("build", "ao_rays", "ao_rays_wide", "ao_rays_wide_quantised", "trace_wide_closest",
                 "camera_replay_lbvh", "camera_replay_ploc", "batch_trace", "pt", "adjoint")


def profile_case(name, dev):
    """One small case of one kernel for an ncu capture: the set-up, then the
    kernel's launch chain twice (capture the second launch: ncu -s 1 -c 1 -k
    <kernel>), with the inputs larger than L2 and a few GB on the device at
    most. No timing; prints what ran.
      build                   4M-triangle soup: the build chain (k_scene_bounds,
                              k_keys, 4 x sort::k_onesweep, k_build)
      ao_rays                 4M soup, one 1920x1080 AO frame (64 rays of
                              radius 0.1): k_ao_primary, k_ao_rays, k_ao_finish
      ao_rays_wide(_quantised) the same frame over the 4-wide tree (its
                              8-bit slots)
      trace_wide_closest      4M soup, 1M camera rays closest-hit over the
                              quantised 4-wide slots (k_trace_wide)
      camera_replay_lbvh/_ploc 4M soup, the same camera rays closest-hit on the
                              replay walk (k_trace) over the LBVH / the PLOC tree
      batch_trace             48 meshes of the batched workload (64..262,144
                              triangles, 4,096..1M rays each): k_batch_trace
      pt                      heightfield + icospheres, one 512x512 path-tracing
                              pass (k_pt, stack-free walk)
      adjoint                 the differentiation workload (512x512, 64 spp, 3
                              bounces): k_pt_diff_render, k_pt_diff_adjoint"""
    import torch
    import minimumlbvh_b200 as mb
    from minimumlbvh_b200 import scenes
    if name in ("build", "ao_rays", "ao_rays_wide", "ao_rays_wide_quantised", "trace_wide_closest",
                "camera_replay_lbvh", "camera_replay_ploc"):
        wl = WORKLOADS["soup4m_ao64"]
        tris, (eye, c, up, fovy) = make_scene(wl)
        n, w, h = len(tris), wl["w"], wl["h"]
        d_tris = torch.from_numpy(tris).to(dev)
        b = mb.BVHGPUBuilder()
        sorter = mb.OnesweepSort(dev.index)
        cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
        if name == "camera_replay_ploc":
            b.buildByPLOC(d_tris, n, 0, sorter, 8)
        else:
            b.build(d_tris, n, 0, sorter)
        b.status()
        px = torch.zeros(w * h, dtype=torch.int32, device=dev)
        wide = None
        if name.startswith("ao_rays_wide") or name == "trace_wide_closest":
            wide = mb.WideBVH.from_builder(b, d_tris).quantise()
        rays = None
        if name == "trace_wide_closest" or name.startswith("camera_replay"):
            rays = torch.from_numpy(scenes.camera_rays(cam.m_origin, cam.m_right, cam.m_up, w, h, 2)).to(dev)
        for _ in range(2):
            if name == "build":
                b.build(d_tris, n, 0, sorter)
            elif name == "ao_rays":
                mb.render_ao(px, (w, h), cam, b.m_rootNode, b.m_internals, d_tris, 1, wl["ns"], wl["radius"], 12345)
            elif name == "trace_wide_closest":
                mb.intersect_wide(wide, rays, quantised=True, rayQuery=mb.RAY_QUERY_CLOSEST)
            elif name.startswith("camera_replay"):
                mb.intersect(b, d_tris, rays, traversal=mb.TRAVERSAL_REPLAY)
            else:
                mb.render_ao_wide(px, (w, h), cam, wide, 1, wl["ns"], wl["radius"], 12345,
                                  quantised=name.endswith("quantised"))
        b.status()
    elif name == "batch_trace":
        tris, offsets = scenes.batched_soup(48, 64, 262_144, seed=7, device=dev)
        rays, roff = scenes.batched_rays(tris, offsets, 4096, 1_048_576, seed=8)
        bb = mb.BatchedBVH(tris, torch.as_tensor(offsets.astype(np.int32), device=dev), len(offsets) - 1)
        bb.set_rays(rays, torch.as_tensor(roff.astype(np.int32), device=dev))
        bb.build()
        for _ in range(2):
            bb.trace()
        bb.status()
        n = int(offsets[-1])
    elif name == "pt":
        tris = scenes.heightfield_icospheres()
        n = len(tris)
        t = torch.from_numpy(tris).to(dev)
        at = torch.from_numpy(scenes.pt_attributes(n)).to(dev)
        b = mb.BVHGPUBuilder().build(t, n, 0, mb.OnesweepSort(dev.index))
        eye, c, up, fovy = scenes.camera_heightfield()
        cam = mb.RayGenerator().lookat(eye, c, up, fovy, 512, 512)
        acc = torch.zeros(512 * 512 * 4, dtype=torch.float32, device=dev)
        for _ in range(2):
            mb.render_pt(acc, (512, 512), cam, b.m_rootNode, b.m_internals, t, at)
        b.status()
    elif name == "adjoint":
        tris, alb, em = scenes.diff_scene()
        n = len(tris)
        t = torch.from_numpy(tris).to(dev)
        b = mb.BVHGPUBuilder().build(t, n, 0, mb.OnesweepSort(dev.index))
        eye, c, up, fovy = scenes.camera_heightfield()
        cam = mb.RayGenerator().lookat(eye, c, up, fovy, 512, 512)
        a = torch.from_numpy(alb).to(dev)
        e = torch.from_numpy(em).to(dev)
        img = torch.empty(512 * 512, dtype=torch.float32, device=dev)
        grad = torch.zeros(n, dtype=torch.float32, device=dev)
        for _ in range(2):
            mb.pt_diff_render(img, (512, 512), cam, b, t, a, e, 64, 3)
            mb.pt_diff_adjoint(grad, img, (512, 512), cam, b, t, a, e, 64, 3)
        b.status()
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": name, "triangles": n, "device_bytes": torch.cuda.max_memory_allocated(dev)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="soup4m_ao64", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=8.0, help="wall time of the CPU-baseline AO sample")
    ap.add_argument("--ref-seconds", type=float, default=4.0, help="wall time of one reference-arm step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--image", default=None, help="override the frame size, WxH (small cases for ncu captures)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (1,024-mesh) workload")
    ap.add_argument("--batched-meshes", type=int, default=1024, help="meshes of the batched workload (small cases)")
    ap.add_argument("--no-autotune", action="store_true", help="batched workload with default launch parameters")
    ap.add_argument("--no-ploc", action="store_true", help="skip the higher-quality (PLOC) build section")
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable path-tracing section")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the baseline leg running the reference's own GPU kernels")
    ap.add_argument("--profile-case", choices=PROFILE_CASES, default=None,
                    help="run one small case of one kernel for an ncu capture (no timing) and exit")
    args = ap.parse_args()
    if args.profile_case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        profile_case(args.profile_case, torch.device("cuda", torch.cuda.current_device()))
        return
    wl = dict(WORKLOADS[args.workload])
    if args.image:
        wl["w"], wl["h"] = (int(v) for v in args.image.lower().split("x"))
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, wl, rank)
        return

    import torch
    import minimumlbvh_b200 as mb

    from minimumlbvh_b200.replicas import Replicas

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    reps = Replicas("nccl", device=dev)
    barrier, max_over_ranks = reps.barrier, reps.max

    tris, (eye, c, up, fovy) = make_scene(wl)
    n, w, h = len(tris), wl["w"], wl["h"]
    host_tris = torch.from_numpy(tris).pin_memory()
    d_tris = host_tris.to(dev)
    builder = mb.BVHGPUBuilder()
    sorter = mb.OnesweepSort(local)
    cam = mb.RayGenerator().lookat(eye, c, up, fovy, w, h)
    pixels = torch.zeros(w * h, dtype=torch.int32, device=dev)
    host_pixels = torch.empty(w * h, dtype=torch.int32).pin_memory()
    stats = torch.zeros(8, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream()

    def ao_frame(with_stats=False, tris_buf=None, out=None):
        mb.render_ao(pixels if out is None else out, (w, h), cam, builder.m_rootNode, builder.m_internals,
                     d_tris if tris_buf is None else tris_buf, 1, wl["ns"], wl["radius"], 12345,
                     stats=stats if with_stats else None)

    # counting pass: rays, node visits and triangle tests of one frame (the
    # traversal is deterministic, so every timed frame does the same work)
    builder.build(d_tris, n, 0, sorter)
    builder.status()
    ao_frame(with_stats=True)
    torch.cuda.synchronize()
    st = stats.cpu().numpy()
    rays_per_frame, visits, tests, ao_visits, ao_tests = (int(x) for x in st[:5])
    primaries = w * h
    ao_rays = rays_per_frame - primaries

    for _ in range(args.warmup):
        builder.build(d_tris, n, 0, sorter)
        ao_frame()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    with sampler:
        # ---- AO frames over the resident BVH (inputs > L2: 419 MB working set for the soup)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if wl["scene"] != "soup" else None
        barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            if flush is not None:
                flush.zero_()  # evict the L2-resident scene between frames
            ev[i][0].record(stream)
            mb.profile_events(*kev[i])
            ao_frame()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        ao_ms = [a.elapsed_time(b) for a, b in ev]
        kernel_ms = [a.elapsed_time(b) for a, b in kev]
        ao_total_s = max_over_ranks(sum(ao_ms) / 1e3)

        # ---- the other forms, at equal results: the replay walk over the same
        # FP32 nodes, and the replay walk over the 8-bit quantised tree
        qtree = mb.QuantisedBVH.from_builder(builder, d_tris)
        occ_plain = torch.empty(w * h, dtype=torch.int32, device=dev)
        mb.render_ao(pixels, (w, h), cam, builder.m_rootNode, builder.m_internals, d_tris, 1, wl["ns"], wl["radius"],
                     12345, occluded=occ_plain)

        leaf_tris = mb.leaf_triangles(builder, d_tris)

        def replay_frame(occluded=None, stats=None):
            mb.render_ao(pixels, (w, h), cam, builder.m_rootNode, builder.m_internals, d_tris, 1, wl["ns"],
                         wl["radius"], 12345, occluded=occluded, stats=stats, traversal=mb.TRAVERSAL_REPLAY,
                         leaf_triangles=leaf_tris)

        def quantised_frame(occluded=None, stats=None):
            mb.render_ao_quantised(pixels, (w, h), cam, qtree, 1, wl["ns"], wl["radius"], 12345, occluded=occluded,
                                   stats=stats)

        # the 4-wide tree for the AO rays: regrouping + leaf-ordered triangles,
        # timed as the form's preparation per build
        wide = mb.WideBVH.from_builder(builder, d_tris)
        wev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            wev[i][0].record(stream)
            wide.update(stream)
            wev[i][1].record(stream)
        torch.cuda.synchronize()
        wide_prep_ms = float(np.mean([a.elapsed_time(b) for a, b in wev]))

        def wide_frame(occluded=None, stats=None):
            mb.render_ao_wide(pixels, (w, h), cam, wide, 1, wl["ns"], wl["radius"], 12345, occluded=occluded,
                              stats=stats)

        # its 8-bit quantised slots (64 bytes instead of 128)
        wide.quantise()
        qev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            qev[i][0].record(stream)
            wide.quantise(stream)
            qev[i][1].record(stream)
        torch.cuda.synchronize()
        wide_quant_ms = float(np.mean([a.elapsed_time(b) for a, b in qev]))
        quant_status = int(wide.status[0].item())

        def wide_quantised_frame(occluded=None, stats=None):
            mb.render_ao_wide(pixels, (w, h), cam, wide, 1, wl["ns"], wl["radius"], 12345, occluded=occluded,
                              stats=stats, quantised=True)

        forms = {}
        form_occ_host = {}
        occ_plain_host = occ_plain.cpu().numpy().view(np.uint32)
        for name, frame in (("replay", replay_frame), ("quantised", quantised_frame), ("wide", wide_frame),
                            ("wide_quantised", wide_quantised_frame)):
            occ = torch.empty_like(occ_plain)
            fst = torch.zeros(8, dtype=torch.int64, device=dev)
            frame(occluded=occ, stats=fst)
            for _ in range(args.warmup):
                frame()
            fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            fkev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                    for _ in range(args.steps)]
            barrier()
            torch.cuda.synchronize()
            for i in range(args.steps):
                if flush is not None:
                    flush.zero_()
                fev[i][0].record(stream)
                mb.profile_events(*fkev[i])
                frame()
                fev[i][1].record(stream)
            torch.cuda.synchronize()
            barrier()
            forms[name] = (max_over_ranks(sum(a.elapsed_time(b) for a, b in fev) / 1e3),
                           float((occ_plain == occ).double().mean().item()), fst.cpu().numpy(),
                           float(np.mean([a.elapsed_time(b) for a, b in fkev])) / 1e3)
            form_occ_host[name] = occ.cpu().numpy().view(np.uint32)

        # ---- builds
        bev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        barrier()
        torch.cuda.synchronize()
        cbev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
        for i in range(args.steps):
            if flush is not None:
                flush.zero_()
            bev[i][0].record(stream)
            mb.profile_events(*cbev[i])  # around the agglomerative climb (k_build)
            builder.build(d_tris, n, 0, sorter)
            bev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        climb_ms = float(np.mean([a.elapsed_time(b) for a, b in cbev]))
        build_ms = [a.elapsed_time(b) for a, b in bev]
        build_total_s = max_over_ranks(sum(build_ms) / 1e3)
        builder.status()

        # ---- the higher-quality (PLOC) build and the forms over its tree
        lbvh_forms = {"build_ms": build_total_s * 1e3 / args.steps, "rays_per_frame": rays_per_frame,
                      "plain": ao_total_s * 1e3 / args.steps, "replay": forms["replay"][0] * 1e3 / args.steps,
                      "wide": forms["wide"][0] * 1e3 / args.steps}
        ploc = None if args.no_ploc else bench_ploc(args, wl, d_tris, n, cam, w, h, dev, stream, barrier,
                                                    max_over_ranks, flush, builder, lbvh_forms, occ_plain)

        # ---- end to end through the C ABI from host buffers: every step uploads
        # its triangles from pinned host memory, builds, renders and reads the
        # image back. Two device triangle buffers: step i + 1's upload (copy
        # stream) overlaps step i's build and frame; a buffer is refilled only
        # after the step that read it is done. Two image buffers: step i's
        # read-back (a second copy stream) overlaps step i + 1; an image buffer
        # is rendered into again only after its read-back is done. The timed
        # region ends after the last read-back.
        eev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        copy_stream = torch.cuda.Stream(device=dev)
        d2h_stream = torch.cuda.Stream(device=dev)
        bufs = (d_tris, torch.empty_like(d_tris))
        pix = (pixels, torch.zeros_like(pixels))
        hpix = (host_pixels, torch.empty_like(host_pixels).pin_memory())

        def read_back(i, done):
            d2h_stream.wait_event(done[i])
            with torch.cuda.stream(d2h_stream):
                hpix[i % 2].copy_(pix[i % 2], non_blocking=True)
            read[i].record(d2h_stream)

        ready = [torch.cuda.Event() for _ in range(args.steps)]
        done = [torch.cuda.Event() for _ in range(args.steps)]
        read = [torch.cuda.Event() for _ in range(args.steps)]
        barrier()
        torch.cuda.synchronize()
        eev[0].record(stream)
        copy_stream.wait_event(eev[0])
        for i in range(args.steps):
            buf = bufs[i % 2]
            if i >= 2:
                copy_stream.wait_event(done[i - 2])
            with torch.cuda.stream(copy_stream):
                buf.copy_(host_tris, non_blocking=True)
            ready[i].record(copy_stream)
            stream.wait_event(ready[i])
            if i >= 2:
                stream.wait_event(read[i - 2])
            builder.build(buf, n, 0, sorter)
            ao_frame(tris_buf=buf, out=pix[i % 2])
            done[i].record(stream)
            read_back(i, done)
        stream.wait_event(read[args.steps - 1])
        eev[1].record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_s = max_over_ranks(eev[0].elapsed_time(eev[1]) / 1e3)

        # ---- the same end to end with the chosen form: every step also
        # regroups the new tree 4-wide (slots + leaf-ordered triangles) and
        # renders its AO rays over it; one wide tree per triangle buffer
        wides = [mb.WideBVH.from_builder(builder, b) for b in bufs]
        cev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ready = [torch.cuda.Event() for _ in range(args.steps)]
        done = [torch.cuda.Event() for _ in range(args.steps)]
        read = [torch.cuda.Event() for _ in range(args.steps)]
        barrier()
        torch.cuda.synchronize()
        cev[0].record(stream)
        copy_stream.wait_event(cev[0])
        for i in range(args.steps):
            buf = bufs[i % 2]
            if i >= 2:
                copy_stream.wait_event(done[i - 2])
            with torch.cuda.stream(copy_stream):
                buf.copy_(host_tris, non_blocking=True)
            ready[i].record(copy_stream)
            stream.wait_event(ready[i])
            if i >= 2:
                stream.wait_event(read[i - 2])
            builder.build(buf, n, 0, sorter)
            wides[i % 2].update(stream)
            mb.render_ao_wide(pix[i % 2], (w, h), cam, wides[i % 2], 1, wl["ns"], wl["radius"], 12345)
            done[i].record(stream)
            read_back(i, done)
        stream.wait_event(read[args.steps - 1])
        cev[1].record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_chosen_s = max_over_ranks(cev[0].elapsed_time(cev[1]) / 1e3)
        del wides
        builder.build(d_tris, n, 0, sorter)
        precision = bench_precision(args, builder, qtree, wide, d_tris, tris, cam, w, h, dev, stream, max_over_ranks)
        precision["heightfield"] = bench_precision_heightfield(args, dev, stream, max_over_ranks)
        pt = bench_pt(args, dev, stream, max_over_ranks,
                      reference_gpu=not args.no_reference_gpu and rank == 0 and world == 1)
        diff = None if args.no_diff else bench_diff(args, dev, stream, max_over_ranks)
        reference_gpu = None
        if not args.no_reference_gpu and rank == 0 and world == 1:
            reference_gpu = bench_reference_gpu(args, builder, sorter, d_tris, n, cam, w, h, dev, stream,
                                                lambda x: x)
        batched = None if args.no_batched else bench_batched(args, dev, stream, barrier, max_over_ranks,
                                                                   world, args.batched_meshes, not args.no_autotune)
        onchip = onchip_peaks(dev, stream)
    clocks = sampler.summary()

    ms_per_step = ao_total_s * 1e3 / args.steps
    value = rays_per_frame * args.steps * world / ao_total_s / 1e6
    kernel_avg_s = float(np.mean(kernel_ms)) / 1e3
    peak, peak_kind = peaks()
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, no dataset)",
        "config": {"workload": args.workload, "triangles": n, "image": [w, h], "ao_samples": wl["ns"],
                   "ao_radius": wl["radius"], "rays_per_frame": rays_per_frame, "primary_rays": primaries,
                   "ao_rays": ao_rays, "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (nodes + triangles 419 MB)" if wl["scene"] == "soup"
                   else "L2 flushed (256 MB write) between timed frames"},
        "gpu_launches": args.steps * (3 + 3 + 3 + 3 + 3 + 2 + 1 + 7 + 10 + 12),  # AO, replay, quantised, wide, wide
        # quantised AO, wide prep, quantisation,
        # build, e2e steps, chosen-form e2e steps (7 build + 2 prep + 3 AO)
        "clocks": clocks,
    }
    # roofline of the dominant kernel (k_ao_rays): algorithmic bytes of its rays
    # (64 B per internal-node visit + 36 B per triangle test, counted by the
    # deterministic counting pass) over its event-timed duration per launch
    kernel_bytes = 64 * ao_visits + 36 * ao_tests
    achieved = kernel_bytes / kernel_avg_s / 1e9
    traffic = committed_traffic(args.workload)
    # The kernel's bytes are served on chip (L1 and L2 hits; its DRAM traffic
    # is a fraction of a percent of them), so its roofline is the on-chip
    # bandwidth of its own load pattern: 32-byte sectors gathered at random
    # from an L2-resident buffer, measured by this project's probe kernel.
    # The HBM copy bandwidth is kept as the denominator of its DRAM traffic.
    onchip_peak = onchip["l2_gather_gbs"]
    line["roofline"] = {"bound": "l2", "achieved": achieved, "peak": onchip_peak, "unit": "GB/s",
                        "frac": achieved / onchip_peak, "traffic": traffic, "kernel": "k_ao_rays",
                        "kernel_ms": kernel_avg_s * 1e3,
                        "peak_source": "builder-measured: mlbvh_read_probe gathering random 32-byte sectors from a "
                                       "64 MiB L2-resident buffer (the traversal's load), CUDA events",
                        "frac_of_l2_stream": achieved / onchip["l2_stream_gbs"],
                        "hbm": {"peak": peak, "peak_source": f"{peak_kind} hbm_gbs",
                                "traffic_gbs": (traffic / kernel_avg_s / 1e9) if traffic else None,
                                "frac": (traffic / kernel_avg_s / 1e9 / peak) if traffic else None},
                        "onchip_peaks": onchip,
                        "bytes_model": "64 B per internal-node visit + 36 B per triangle test",
                        "node_visits_per_ray": visits / rays_per_frame, "tri_tests_per_ray": tests / rays_per_frame,
                        "kernel_bytes": kernel_bytes}
    build_s = build_total_s / args.steps
    line["build"] = {"ms": build_s * 1e3, "climb_ms": climb_ms, "mtri_s": n * world / build_s / 1e6,
                     "achieved_gbs": n * BUILD_BYTES_PER_TRI / build_s / 1e9,
                     "frac": n * BUILD_BYTES_PER_TRI / build_s / 1e9 / peak, "bytes_per_tri": BUILD_BYTES_PER_TRI}
    line["e2e"] = {"value": rays_per_frame * args.steps * world / e2e_s / 1e6, "unit": "Mrays/s",
                   "h2d_bytes_per_step": int(host_tris.numel() * 4), "d2h_bytes_per_step": int(w * h * 4),
                   "ms_per_step": e2e_s * 1e3 / args.steps,
                   "pipeline": "upload of step i+1 overlaps build + frame of step i (two device triangle buffers); read-back of step i overlaps step i+1 (two image buffers)"}
    line["e2e_chosen"] = {"value": rays_per_frame * args.steps * world / e2e_chosen_s / 1e6, "unit": "Mrays/s",
                          "h2d_bytes_per_step": int(host_tris.numel() * 4), "d2h_bytes_per_step": int(w * h * 4),
                          "ms_per_step": e2e_chosen_s * 1e3 / args.steps,
                          "form": "the chosen form end to end: upload, build, 4-wide regrouping + leaf-ordered "
                                  "triangles, AO frame over the wide tree, image download (same pipelining)"}
    form_lines = {}
    form_desc = {
        "replay": "FP32 nodes, replay walk (stack of pending far children), leaf-ordered 48-byte triangles",
        "quantised": "quantised 8-bit child boxes (32-byte nodes), replay walk",
        "wide": "AO rays over the 4-wide regrouping of the FP32 tree (128-byte nodes, any-hit), "
                "primary rays on the replay walk, leaf-ordered 48-byte triangles",
        "wide_quantised": "AO rays over the 4-wide tree with 8-bit child planes rounded outward (64-byte nodes, "
                          "any-hit, exact leaf-box check on hits), primary rays on the replay walk",
    }
    for name, (total_s, agree, fst, f_kernel_s) in forms.items():
        f_rays = int(fst[0])
        if name == "replay":
            node_bytes = 64 * int(fst[1])
        elif name == "quantised":
            node_bytes = 32 * int(fst[1]) + 4 * int(fst[5])
        else:  # primary rays visit 64-byte binary nodes, AO rays 128-byte (64-byte quantised) wide nodes
            node_bytes = 64 * (int(fst[1]) - int(fst[3])) + (128 if name == "wide" else 64) * int(fst[3])
        tri_bytes = 48 * int(fst[2])
        # the AO-ray kernel of this form: its algorithmic bytes (node bytes of
        # its AO-ray visits + 48 B per AO-ray triangle test) per launch over its
        # event-timed duration
        if name == "replay":
            ao_node_bytes = 64 * int(fst[3])
        elif name == "quantised":
            ao_node_bytes = 32 * int(fst[3]) + 4 * int(fst[6])
        else:
            ao_node_bytes = (128 if name == "wide" else 64) * int(fst[3])
        f_kernel_bytes = ao_node_bytes + 48 * int(fst[4])
        f_achieved = f_kernel_bytes / f_kernel_s / 1e9
        form_lines_roof = {"kernel_ms": f_kernel_s * 1e3, "achieved": f_achieved, "peak": onchip_peak,
                           "unit": "GB/s", "frac": f_achieved / onchip_peak, "kernel_bytes": f_kernel_bytes}
        form_lines[name] = {
            "form": form_desc[name],
            "value": f_rays * args.steps * world / total_s / 1e6, "unit": "Mrays/s",
            "ms_per_step": total_s * 1e3 / args.steps, "vs_plain": ao_total_s / total_s,
            "occlusion_agreement": agree, "rays_per_frame": f_rays,
            "node_visits_per_ray": int(fst[1]) / max(f_rays, 1),
            "node_bytes_per_ray": node_bytes / max(f_rays, 1), "tri_bytes_per_ray": tri_bytes / max(f_rays, 1),
            "ao_kernel_roofline": form_lines_roof}
        if name == "wide":
            form_lines[name]["prep_ms_per_build"] = wide_prep_ms
            form_lines[name]["restarts"] = int(fst[6])
        if name == "wide_quantised":
            form_lines[name]["prep_ms_per_build"] = wide_prep_ms + wide_quant_ms
            form_lines[name]["restarts"] = int(fst[6])
            form_lines[name]["quantisation_status"] = quant_status
    exact = [k for k, v in form_lines.items() if v["occlusion_agreement"] == 1.0]
    best = max(exact, key=lambda k: form_lines[k]["value"]) if exact else None
    line["chosen"] = dict(form_lines[best]) if best else {"form": None, "note": "no form agreed with the plain one"}
    line["chosen"]["plain_node_visits_per_ray"] = visits / max(rays_per_frame, 1)
    line["chosen"]["plain_node_bytes_per_ray"] = 64 * visits / max(rays_per_frame, 1)
    line["forms"] = form_lines
    line["precision"] = precision
    line["gpu_launches"] += precision["launches"] + precision["heightfield"]["launches"]
    line["pt"] = pt
    if ploc is not None:
        line["ploc"] = ploc
        line["gpu_launches"] += ploc["launches"]
    if diff is not None:
        line["differentiation"] = diff
        line["gpu_launches"] += diff["launches"]
    line["gpu_launches"] += 2 * (args.warmup + args.steps) + 8  # pt passes, its build and leaf copy
    if "ploc_replay" in pt:
        line["gpu_launches"] += (args.warmup + args.steps) + 9  # PLOC pt passes, its build and leaf copy
    if reference_gpu is not None:
        line["reference_gpu_baseline"] = reference_gpu
        if "ao" in reference_gpu:  # our kernels launched in that leg: plain (3) and wide (3) frames, 2 builds
            line["gpu_launches"] += (args.warmup + args.steps) * (3 + 3 + 7) + 2
    line["gpu_launches"] += 2 * (args.warmup + args.steps) + 1
    line["gpu_launches"] += onchip["launches"]
    if batched is not None:
        line["batched"] = batched
        line["gpu_launches"] += batched["launches"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out = {"nodes": builder.m_internals.cpu().numpy().view(np.uint32)[: n - 1],
               "root": int(builder.m_rootNode.cpu().numpy().view(np.uint32)[0])}
        cam_arr = cam.as_array()
        cb, _, occ_ref = cpu_sample_ao(wl, tris, cam_arr, out, args.cpu_seconds, rows=cpu_rows(wl))
        cb["build"] = cpu_build_baseline(tris)
        line["cpu_baseline"] = cb
        line["occlusion_agreement_vs_oracle"] = oracle_agreement(wl, tris, cam_arr, out, occ_plain_host,
                                                                 form_occ_host, occ_ref, cb["kind"])
    reps.close()
    if reps.is_root:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
