"""The BFS level loop on the device (one CUDA graph per search: WHILE {decide;
SWITCH {push per warp | balanced push | pull}}) against the host-driven loop
and the oracle: the same distances, `reachable` and `max_depth`, with the
fixed rule and with the learned schedule, on symmetric graphs (all three
variants) and directed CSRs (pushes only), for repeated searches on one graph
(the graph is built once and relaunched), and after the schedule changes
(the graph is rebuilt)."""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import schedule as sched
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def both_loops(device, g, sources):
    out = {}
    for on in (True, False):
        device.set_bfs_device_loop(on)
        out[on] = [g.bfs_array(int(s)) for s in sources]
    device.set_bfs_device_loop(True)
    return out[True], out[False]


def check(device, o, t, sources, label):
    g = G.GpuGraph.from_csr(o, t, device)
    dev_runs, host_runs = both_loops(device, g, sources)
    for s, a, b in zip(sources, dev_runs, host_runs):
        ref = O.bfs(o, t, int(s))
        assert np.array_equal(a["distances"], ref["distances"]), (label, int(s))
        assert np.array_equal(b["distances"], ref["distances"]), (label, int(s))
        assert (a["reachable"], a["max_depth"]) == (ref["reachable"], ref["max_depth"]), (label, int(s))
        assert (b["reachable"], b["max_depth"]) == (ref["reachable"], ref["max_depth"]), (label, int(s))


def graphs():
    out = []
    for scale, seed in ((10, 1), (14, 3), (17, 2)):
        c = G.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
        out.append((f"rmat{scale}", c.offsets, c.targets))
    c = G.generate_erdos_renyi(1 << 15, 8 << 15, seed=3)
    out.append(("er15", c.offsets, c.targets))
    # A long path with side branches: many levels, small frontiers.
    n = 5000
    pairs = [(i, i + 1) for i in range(n - 1)] + [(i, n + i) for i in range(0, n, 7)]
    c = G.from_edge_pairs(pairs, n + n, True)
    out.append(("path", c.offsets, c.targets))
    # Directed (non-symmetric) CSR: pushes only.
    rng = np.random.default_rng(4)
    c = G.from_edge_pairs(rng.integers(0, 3000, size=(20000, 2)), 3000, False)
    out.append(("directed", c.offsets, c.targets))
    return out


def test_device_loop_matches_host_loop_and_oracle(device):
    for label, o, t in graphs():
        deg = np.diff(o)
        live = np.flatnonzero(deg > 0)
        rng = np.random.default_rng(len(o))
        sources = list(rng.choice(live, size=min(6, len(live)), replace=False)) + [int(np.argmin(deg))]
        check(device, o, t, sources, label)


def test_device_loop_with_the_learned_schedule(device):
    import os

    if not os.path.exists(sched.DEFAULT_WEIGHTS):
        pytest.skip("no shipped schedule network")
    c = G.generate_rmat(16, 16, 0.57, 0.19, 0.19, seed=7)
    g = G.GpuGraph.from_csr_arrays(c, device)
    sources = [0, 5, 1000, 40000]
    plain = [g.bfs_array(s)["distances"] for s in sources]  # builds the fixed-rule graph
    sched.install(device)  # the loop graph is rebuilt with the network
    try:
        dev_runs, host_runs = both_loops(device, g, sources)
    finally:
        device.set_schedule(None)
    for s, p, a, b in zip(sources, plain, dev_runs, host_runs):
        ref = O.bfs(c.offsets, c.targets, s)
        assert np.array_equal(a["distances"], ref["distances"]) and np.array_equal(p, ref["distances"]), s
        assert np.array_equal(b["distances"], ref["distances"]), s
        assert a["max_depth"] == b["max_depth"] == ref["max_depth"]
    # back on the fixed rule (rebuilt again)
    assert np.array_equal(g.bfs_array(5)["distances"], plain[1])
