"""bench.py pieces that run without a GPU: the surface-area cost it reports
for the PLOC section (a torch computation, run here on CPU tensors) against
the oracle's, and the reference arm's JSON line (the reference's own CPU
code; every key the driver reads)."""
import json
import os
import subprocess
import sys

import numpy as np

import _oracle as O
from minimumlbvh_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sah_cost_matches_oracle():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    tris = scenes.gaussian_soup(20000, clusters=8, seed=5)
    for out in (O.build(tris), O.build_ploc(tris, 0, 8)):
        nodes = torch.from_numpy(out["nodes"].view(np.int32).copy())
        root = torch.tensor([out["root"]], dtype=torch.int64)
        got = bench.sah_cost_device(nodes, root)
        np.testing.assert_allclose(got, O.sah_cost(out["nodes"], out["root"]), rtol=1e-9)


def test_reference_arm_line():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ref-seconds", "1"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config", "cpu_baseline",
                "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
