"""Learned schedule: traces, training and evaluation of the schedule network.

The network (12 features -> 32 -> 32 -> 3 predicted log2 microseconds, BF16
weights, FP32 accumulation; csrc/sched.cuh) picks the step variant of every
BFS level (warp-per-vertex push, load-balanced push, pull) and the
intersection variant of every out-degree bucket of the triangle count (warp
hash table, CTA hash table, CTA binary search). It only changes which kernels
run, never a result, and the fixed rules (alpha/beta direction, degree-range
buckets) stay its fallback.

Everything here runs on the GPU through the library: the training graphs are
generated on the device, the plain kernels emit the traces (every valid
variant timed from the same state), and the network is trained by the
project's own forward/backward/Adam kernels.

    python -m grafeo_cuda.schedule train --graphs 2000 --heldout 200 --out weights.json

Training corpus (seeded): R-MAT scale 16-22 with a ~ U[0.45, 0.65],
b = c = (0.95 - a) / 2, edge factor 16; 2D grids with 5% edge dropout and
sides in [256, 2048]; random geometric graphs with 2^16..2^21 points and
average degree U[8, 64]. Held-out graphs use seeds the training set never
draws.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

import grafeo_cuda as G

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "schedule_weights.json")
HELDOUT_SEED_BASE = 1_000_000  # held-out graph seeds start here; training seeds stay below


# ---------------------------------------------------------------- corpus


# The device's kSchedMarginLog2 (csrc/sched.cuh): the learned pick must be
# predicted at least 2^MARGIN_LOG2 faster than the fixed rule's variant.
MARGIN_LOG2 = 0.2


def corpus(count: int, seed: int, scale_range=(16, 22)) -> list[dict]:
    """Seeded graph specs, one quarter each R-MAT, grid, geometric and
    Erdos-Renyi (uniform neighbours: no hubs and no locality)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        kind = ("rmat", "grid", "geometric", "erdos_renyi")[i % 4]
        gseed = int(seed * 100_003 + i)
        if kind == "rmat":
            a = float(rng.uniform(0.45, 0.65))
            specs.append({"kind": kind, "scale": int(rng.integers(scale_range[0], scale_range[1] + 1)),
                          "a": a, "b": (0.95 - a) / 2, "c": (0.95 - a) / 2, "seed": gseed})
        elif kind == "grid":
            lo, hi = 2 ** (scale_range[0] // 2), 2 ** ((scale_range[1] + 1) // 2)
            specs.append({"kind": kind, "width": int(rng.integers(lo, hi + 1)), "height": int(rng.integers(lo, hi + 1)),
                          "drop": 0.05, "seed": gseed})
        elif kind == "geometric":
            specs.append({"kind": kind, "n": int(2 ** rng.integers(scale_range[0], scale_range[1])),
                          "avg_degree": float(rng.uniform(8, 64)), "seed": gseed})
        else:
            n = int(2 ** rng.integers(scale_range[0], scale_range[1] + 1))
            specs.append({"kind": kind, "n": n, "pairs": int(n * rng.uniform(4, 32)), "seed": gseed})
    return specs


def make_graph(device: G.GpuDevice, spec: dict) -> G.GpuGraph:
    k = spec["kind"]
    if k == "rmat":
        return G.GpuGraph.generate_rmat(device, spec["scale"], 16, spec["a"], spec["b"], spec["c"], spec["seed"])
    if k == "grid":
        return G.GpuGraph.generate_grid(device, spec["width"], spec["height"], spec["drop"], spec["seed"])
    if k == "geometric":
        return G.GpuGraph.generate_geometric(device, spec["n"], spec["avg_degree"], spec["seed"])
    if k == "erdos_renyi":
        return G.GpuGraph.generate_erdos_renyi(device, spec["n"], spec["pairs"], spec["seed"])
    raise ValueError(f"unknown graph kind {k!r}")


def pick_sources(graph: G.GpuGraph, count: int, seed: int) -> list[int]:
    rng = np.random.default_rng(seed)
    return [int(s) for s in rng.integers(0, graph.num_nodes, size=count)]


# ---------------------------------------------------------------- traces


def _targets(times: np.ndarray, valid: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    mask = np.stack([(valid >> c) & 1 for c in range(G.SCHEDULE_OUTPUTS)], axis=1).astype(np.uint8)
    mask &= np.isfinite(times).astype(np.uint8)
    y = np.where(mask.astype(bool), np.log2(np.maximum(np.nan_to_num(times, nan=1.0), 1e-3)), 0.0)
    return y.astype(np.float32), mask


def collect(device: G.GpuDevice, specs: list[dict], sources: int = 2, explore: bool = True,
            tc: bool = True, log=None) -> dict:
    """Traces of every spec: BFS from `sources` random sources (skipping
    isolated ones) and one triangle count."""
    feats, times, valid, fixed, kind, graph_id = [], [], [], [], [], []
    t0 = time.time()
    for gi, spec in enumerate(specs):
        g = make_graph(device, spec)
        got, tries = 0, 0
        for s in pick_sources(g, 8 * sources, spec["seed"]):
            if got == sources:
                break
            tries += 1
            tr = g.bfs_trace(s, explore_seed=spec["seed"] * 31 + s if explore else 0)
            if tr["levels"] == 0:
                continue
            got += 1
            n = len(tr["valid"])
            feats.append(tr["features"])
            times.append(tr["times_us"])
            valid.append(tr["valid"])
            fixed.append(tr["fixed_rule"])
            kind += [0] * n
            graph_id += [gi] * n
        if tc:
            tr = g.triangle_trace()
            n = len(tr["valid"])
            feats.append(tr["features"])
            times.append(tr["times_us"])
            valid.append(tr["valid"])
            fixed.append(tr["fixed_rule"])
            kind += [1] * n
            graph_id += [gi] * n
        del g
        if log and (gi + 1) % 50 == 0:
            log(f"traced {gi + 1}/{len(specs)} graphs, {sum(len(v) for v in valid)} decisions, {time.time() - t0:.0f} s")
    f = np.concatenate(feats) if feats else np.zeros((0, G.SCHEDULE_FEATURES), np.float32)
    t = np.concatenate(times) if times else np.zeros((0, G.SCHEDULE_OUTPUTS), np.float32)
    v = np.concatenate(valid) if valid else np.zeros(0, np.uint8)
    y, mask = _targets(t, v)
    return {"features": f, "times_us": t, "valid": v, "fixed_rule": np.concatenate(fixed) if fixed else v,
            "kind": np.asarray(kind, np.uint8), "graph": np.asarray(graph_id, np.int64), "targets": y, "mask": mask}


# ---------------------------------------------------------------- training


def init_master(seed: int) -> np.ndarray:
    """He-normal weights, zero biases (FP32 master copy)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, math.sqrt(2 / 12), 32 * 12), np.zeros(32),
             rng.normal(0, math.sqrt(2 / 32), 32 * 32), np.zeros(32),
             rng.normal(0, math.sqrt(1 / 32), 3 * 32), np.zeros(3)]
    return np.concatenate(parts).astype(np.float32)


def train(device: G.GpuDevice, data: dict, steps: int = 6000, batch: int = 1024, lr: float = 3e-3,
          seed: int = 0) -> tuple[np.ndarray, float]:
    master = init_master(seed)
    # Start the output biases at the mean target so the first steps fit shape, not offset.
    y, m = data["targets"], data["mask"].astype(bool)
    master[-3:] = float(y[m].mean()) if m.any() else 0.0
    _, w16, loss = G.schedule_train(device, master, data["features"], y, data["mask"], steps, batch, lr, seed)
    return w16, loss


def choose(device: G.GpuDevice, weights, data: dict) -> np.ndarray:
    """The network's pick for every decision as the device makes it: the
    fixed rule where the network abstains (a non-finite prediction) or where
    it predicts its pick less than 2^MARGIN_LOG2 faster than the fixed rule's
    variant."""
    pred = G.schedule_forward(device, weights, data["features"])
    valid = np.stack([(data["valid"] >> c) & 1 for c in range(G.SCHEDULE_OUTPUTS)], axis=1).astype(bool)
    pred = np.where(valid, pred, np.inf)
    pick = np.argmin(pred, axis=1)
    idx = np.arange(len(pick))
    fixed = data["fixed_rule"].astype(np.int64)
    bad = ~np.all(np.isfinite(np.where(valid, pred, 0.0)), axis=1) if len(pick) else np.zeros(0, bool)
    with np.errstate(invalid="ignore"):
        keep = (pick == fixed) | (pred[idx, fixed] - pred[idx, pick] >= MARGIN_LOG2)
    return np.where(bad | ~keep, fixed, pick)


def trace_gain(device: G.GpuDevice, weights, data: dict) -> dict:
    """Sum of the recorded variant times of the network's picks, the fixed
    rule's picks and the best pick, per decision kind (0 = BFS level, 1 =
    triangle bucket), on traces the network was not trained on."""
    pick = choose(device, weights, data)
    t = np.nan_to_num(data["times_us"], nan=np.inf)
    idx = np.arange(len(pick))
    out = {}
    for k, name in ((0, "bfs"), (1, "triangles")):
        sel = data["kind"] == k
        if not sel.any():
            continue
        learned = float(t[idx[sel], pick[sel]].sum())
        fixed = float(t[idx[sel], data["fixed_rule"][sel]].sum())
        best = float(np.min(t[sel], axis=1).sum())
        out[name] = {"decisions": int(sel.sum()), "learned_us": learned, "fixed_us": fixed, "best_us": best,
                     "gain": fixed / learned if learned > 0 else None,
                     "agree_with_fixed": float((pick[sel] == data["fixed_rule"][sel]).mean())}
    return out


def timed_runs(device: G.GpuDevice, weights, specs: list[dict], sources: int = 4) -> dict:
    """Plain against learned, both timed on the device with CUDA events, and
    the results compared: BFS distances and triangle counts must be equal."""
    tot = {"bfs_plain_ms": 0.0, "bfs_learned_ms": 0.0, "tc_plain_ms": 0.0, "tc_learned_ms": 0.0,
           "bfs_runs": 0, "tc_runs": 0, "identical": True}

    def timed(fn):
        device.synchronize()
        device.timer_start()
        r = fn()
        return r, device.timer_stop()

    for spec in specs:
        g = make_graph(device, spec)
        srcs = pick_sources(g, sources, spec["seed"] + 7)
        for arm in ("plain", "learned"):  # warm both paths once
            device.set_schedule(weights if arm == "learned" else None)
            g.bfs_array(srcs[0], copy_result=False)
            g.triangle_count()
        for s in srcs:
            res = {}
            for arm in ("plain", "learned"):
                device.set_schedule(weights if arm == "learned" else None)
                r, ms = timed(lambda: g.bfs_array(s))
                res[arm] = r["distances"]
                tot[f"bfs_{arm}_ms"] += ms
            tot["identical"] &= bool(np.array_equal(res["plain"], res["learned"]))
            tot["bfs_runs"] += 1
        res = {}
        for arm in ("plain", "learned"):
            device.set_schedule(weights if arm == "learned" else None)
            r, ms = timed(g.triangle_count)
            res[arm] = r["total_triangles"]
            tot[f"tc_{arm}_ms"] += ms
        tot["identical"] &= res["plain"] == res["learned"]
        tot["tc_runs"] += 1
        del g
    device.set_schedule(None)
    for k in ("bfs", "tc"):
        tot[f"{k}_gain"] = tot[f"{k}_plain_ms"] / tot[f"{k}_learned_ms"] if tot[f"{k}_learned_ms"] else None
    return tot


# ---------------------------------------------------------------- weights file


def save(path: str, weights, meta: dict) -> None:
    w = np.asarray(weights, dtype=np.uint16)
    with open(path, "w") as fh:
        json.dump({"format": "grafeo-cuda schedule network 12-32-32-3, BF16 bit patterns",
                   "params": int(w.size), "weights": [int(x) for x in w], "meta": meta}, fh, indent=1)
        fh.write("\n")


def load(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    with open(path) as fh:
        doc = json.load(fh)
    w = np.asarray(doc["weights"], dtype=np.uint16)
    if w.size != G.SCHEDULE_PARAMS:
        raise ValueError(f"{path}: {w.size} parameters, expected {G.SCHEDULE_PARAMS}")
    return w


def install(device: G.GpuDevice, path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    """Loads the trained network and installs it on the device."""
    w = load(path)
    device.set_schedule(w)
    return w


# ---------------------------------------------------------------- command line


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="trace, train on the GPU, evaluate on held-out graphs")
    t.add_argument("--graphs", type=int, default=2000)
    t.add_argument("--heldout", type=int, default=200)
    t.add_argument("--timed", type=int, default=30, help="held-out graphs also timed plain vs learned")
    t.add_argument("--sources", type=int, default=2)
    t.add_argument("--scale-min", type=int, default=16)
    t.add_argument("--scale-max", type=int, default=22)
    t.add_argument("--steps", type=int, default=6000)
    t.add_argument("--seed", type=int, default=4)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--report", default=None, help="write the evaluation JSON here too")
    t.add_argument("--save-traces", default=None, help="write the training and held-out traces (.npz)")
    e = sub.add_parser("eval", help="evaluate the shipped (or given) network on held-out graphs, no training")
    e.add_argument("--heldout", type=int, default=200)
    e.add_argument("--timed", type=int, default=30)
    e.add_argument("--sources", type=int, default=2)
    e.add_argument("--scale-min", type=int, default=16)
    e.add_argument("--scale-max", type=int, default=22)
    e.add_argument("--seed", type=int, default=4)
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--report", default=None)
    a = ap.parse_args(argv)

    dev = G.GpuDevice(0)
    log = lambda msg: print(msg, flush=True)  # noqa: E731
    if a.cmd == "eval":
        w16 = load(a.weights)
        held_specs = corpus(a.heldout, HELDOUT_SEED_BASE + a.seed, (a.scale_min, a.scale_max))
        held = collect(dev, held_specs, a.sources, explore=False, log=log)
        report = {"weights": os.path.basename(a.weights), "margin_log2": MARGIN_LOG2,
                  "heldout": {"graphs": a.heldout, "decisions": int(len(held["valid"])),
                              "trace_gain": trace_gain(dev, w16, held)}}
        if a.timed:
            report["heldout"]["timed"] = timed_runs(dev, w16, held_specs[: a.timed])
        log(json.dumps(report, indent=1))
        if a.report:
            with open(a.report, "w") as fh:
                json.dump(report, fh, indent=1)
        return 0
    scales = (a.scale_min, a.scale_max)
    t0 = time.time()
    train_specs = corpus(a.graphs, a.seed, scales)
    held_specs = corpus(a.heldout, HELDOUT_SEED_BASE + a.seed, scales)
    data = collect(dev, train_specs, a.sources, log=log)
    t1 = time.time()
    log(f"training traces: {len(data['valid'])} decisions from {a.graphs} graphs in {t1 - t0:.0f} s")
    held = collect(dev, held_specs, a.sources, explore=False, log=log)
    if a.save_traces:
        np.savez_compressed(a.save_traces, **{f"train_{k}": v for k, v in data.items()},
                            **{f"heldout_{k}": v for k, v in held.items()})
    t2 = time.time()
    w16, loss = train(dev, data, steps=a.steps, seed=a.seed)
    t3 = time.time()
    log(f"trained {a.steps} steps in {t3 - t2:.1f} s, loss {loss:.4f}")
    report = {
        "train": {"graphs": a.graphs, "decisions": int(len(data["valid"])), "loss": loss,
                  "trace_seconds": round(t1 - t0, 1), "train_seconds": round(t3 - t2, 1), "steps": a.steps},
        "heldout": {"graphs": a.heldout, "decisions": int(len(held["valid"])),
                    "loss": G.schedule_gradient(dev, w16, held["features"], held["targets"], held["mask"])[0],
                    "trace_gain": trace_gain(dev, w16, held)},
        "corpus": {"seed": a.seed, "scales": list(scales), "sources_per_graph": a.sources},
    }
    if a.timed:
        report["heldout"]["timed"] = timed_runs(dev, w16, held_specs[: a.timed])
    log(json.dumps(report, indent=1))
    save(a.out, w16, report)
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(report, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
