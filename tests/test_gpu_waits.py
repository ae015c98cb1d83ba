"""Failure detection without a device fault. With the bounded device waits of
the builds cut to a single poll (mlbvh_set_spin_limit, a test hook), waits
give up: the Onesweep look-back of the key sort, and for the PLOC build also
its look-back, grid barriers and placement hand-downs. Each such build must
end (no hang), report MLBVH_ERR_TIMEOUT through mlbvh_scratch_status (a run
whose waits all happened to be met in time must instead be the oracle's
tree), and leave the device usable: the next build with the default limit is
the oracle's tree again."""
import numpy as np
import pytest

import _gpu as G
import _oracle as O
import minimumlbvh_b200 as mb
from minimumlbvh_b200 import scenes

pytestmark = pytest.mark.gpu
TIMEOUT = 3


@pytest.mark.parametrize("kind", ["lbvh", "ploc"])
def test_short_waits_report_timeout_and_device_stays_usable(cuda, kind):
    import torch
    tris = scenes.gaussian_soup(1 << 20, clusters=16, seed=31)
    n = len(tris)
    t = G.dev(tris)
    sorter = mb.OnesweepSort(0)
    ref = O.build(tris) if kind == "lbvh" else O.build_ploc(tris, 0, 8)

    def run():
        b = mb.BVHGPUBuilder()
        if kind == "lbvh":
            b.build(t, n, 0, sorter)
        else:
            b.buildByPLOC(t, n, 0, sorter, 8)
        return b

    def same_as_oracle(b):
        torch.cuda.synchronize()
        nodes = G.host(b.m_internals, np.uint32)[: n - 1]
        return bool((nodes == ref["nodes"]).all()) and int(G.host(b.m_rootNode, np.uint32)[0]) == ref["root"]

    L = mb.lib()
    timeouts = 0
    L.mlbvh_set_spin_limit(1)
    try:
        for _ in range(3):
            b = run()
            try:
                b.status()
            except mb.MlbvhError as e:
                assert e.status == TIMEOUT, e
                timeouts += 1
                continue
            assert same_as_oracle(b), "a build that reported no timeout must be the oracle's tree"
    finally:
        L.mlbvh_set_spin_limit(0)
    # one poll is far shorter than a tile's work: the waits give up
    assert timeouts >= 1
    b = run()
    b.status()
    assert same_as_oracle(b)
