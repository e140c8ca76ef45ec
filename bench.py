#!/usr/bin/env python
"""Benchmark of the four graph hot paths on R-MAT scale 22 (seed 2).

Headline (`metric`/`value`): PageRank iteration throughput in GB/s of
algorithmic traffic, B = 4E + 12V + 4 bytes per iteration (offsets, targets,
one read of the contribution vector and one write of the ranks), on R-MAT
scale 22 (4,194,304 vertices, edge factor 16, a=0.57 b=0.19 c=0.19, seed 2),
50 iterations at damping 0.85 per step. The same JSON line carries BFS
(GTEPS from 64 seeded random non-isolated sources), triangle counting
(edges/s) and k-truss (edges/s, k = 3..8) on the same graph.

  value  device time (CUDA events on the library's stream) with the CSR
         already resident in HBM; inputs (0.53 GB CSR) are larger than L2.
  e2e    the same metric through the public API with host buffers: every step
         copies the CSR from pinned host memory (GpuGraph.from_csr, which also
         validates it), runs pagerank and copies the ranks back.
  roofline  the dominant kernel (one launch = one iteration) against the measured HBM
         copy bandwidth.
  cpu_baseline  the oracle's OpenMP FP64 PageRank on this host's cores, on a
         bounded sample of the same workload.

`--impl reference` times the reference's CPU implementation of the path (the
oracle port; Grafeo's own Rust crate cannot be built here) on the same metric.

Multi-GPU (torchrun): one process per GPU, each a full replica of the graph
running its own PageRank (no data-path collective; weak scaling); value is the
work of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grafeo-cuda_b200"))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, SEED = 22, 16, 2
RMAT_ABC = (0.57, 0.19, 0.19)
DAMPING = 0.85
PR_ITERATIONS = 50
BFS_SOURCES = 64


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--no-secondary", action="store_true", help="skip BFS/TC/k-truss lines")
    ap.add_argument("--suite", action="store_true",
                    help="instead of the headline: all four algorithms on R-MAT 22 and Erdos-Renyi 2^22, and "
                         "R-MAT 24 (directed PageRank with 3%% dangling vertices and its error, truss "
                         "decomposition, BFS and triangles with the learned schedule against the fixed rules); "
                         "one JSON document")
    ap.add_argument("--bfs-breakdown", action="store_true",
                    help="instead of the headline: BFS from 16 random sources on R-MAT 22 and Erdos-Renyi 2^22, "
                         "wall time per search against the sum of its kernels' CUDA-event times (what the per-level "
                         "host round trips cost), per kernel; one JSON document")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed plumbing


class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = True
            self.backend = backend

    def _tensor(self, x):
        import torch

        dev = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch.distributed as dist

        t = self._tensor(x)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch.distributed as dist

        t = self._tensor(x)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ---------------------------------------------------------------- helpers


def pr_bytes(V: int, E: int) -> int:
    return 4 * E + 12 * V + 4


def measured_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name: str):
    """DRAM bytes per launch recorded by the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch_full_size:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = f"/tmp/grafeo_bench_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except OSError:
            return None
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_graph(scale: int):
    import grafeo_cuda as G

    t = time.time()
    csr = G.generate_rmat(scale, EDGE_FACTOR, *RMAT_ABC, seed=SEED)
    return csr, time.time() - t


def pinned_copy(arr: np.ndarray):
    """Copies a u32 array into page-locked host memory (torch pin_memory)."""
    import torch

    t = torch.empty(arr.size, dtype=torch.int32, pin_memory=torch.cuda.is_available())
    view = t.numpy().view(np.uint32)
    view[:] = arr
    return t, view


def bfs_sources(csr, count: int, seed: int) -> np.ndarray:
    deg = np.diff(csr.offsets)
    rng = np.random.default_rng(seed)
    return rng.choice(np.flatnonzero(deg > 0), size=count, replace=False)


def component_edges(csr, dist: np.ndarray) -> int:
    """Undirected edges with both ends in the reached component (Graph500 m)."""
    deg = np.diff(csr.offsets).astype(np.int64)
    return int(deg[dist >= 0].sum() // 2)


# ---------------------------------------------------------------- our implementation


def run_ours(args, d: Dist) -> dict | None:
    import grafeo_cuda as G

    dev = G.GpuDevice(d.local_rank)
    csr, gen_s = make_graph(args.scale)
    V, E = csr.num_nodes, csr.num_edges
    B = pr_bytes(V, E)
    g = G.GpuGraph.from_csr_arrays(csr, dev)

    def pr_step():
        r = g.pagerank_array(DAMPING, PR_ITERATIONS, 0.0, copy_result=False)
        assert r["iterations"] == PR_ITERATIONS

    # -- value: CSR resident in HBM, device time over K steps, max over ranks
    for _ in range(args.warmup):
        pr_step()
    dev.synchronize()
    d.barrier()
    clocks = ClockSampler(d.local_rank)
    clocks.start()
    launches0 = dev.launch_count
    dev.timer_start()
    for _ in range(args.steps):
        pr_step()
    ms = dev.timer_stop()
    launches = dev.launch_count - launches0
    clk = clocks.stop()
    d.barrier()
    ms_max = d.max(ms)
    total_bytes = d.sum(float(B) * PR_ITERATIONS * args.steps)
    value = total_bytes / (ms_max / 1e3) / 1e9

    # -- roofline of the dominant kernel: per-launch device time with events
    dev.set_kernel_timing(True)
    dev.reset_stats()
    pr_step()
    stats = dev.kernel_stats()
    dev.set_kernel_timing(False)
    # The dominant kernel runs once per iteration, so one launch moves B bytes.
    kernel = max(stats, key=lambda k: stats[k][1])
    tile_n, tile_ms = stats[kernel]
    step_ms = sum(v[1] for v in stats.values())
    tile_avg_ms = tile_ms / max(tile_n, 1)
    peak, peak_kind = measured_peak()
    achieved = B / (tile_avg_ms / 1e3) / 1e9
    traffic = profiled_traffic(f"pagerank_{kernel}_rmat22.md")
    roofline = {
        "kernel": kernel,
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": peak,
        "peak_kind": peak_kind,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "frac_of_8tbs_spec": round(achieved / 8000.0, 4),
        "traffic": traffic,
        "algorithmic_bytes_per_launch": B,
        "avg_launch_ms": round(tile_avg_ms, 5),
        "share_of_step": round(tile_ms / step_ms, 4) if step_ms else None,
    }

    # -- e2e through the public API with host buffers
    off_t, off_pinned = pinned_copy(csr.offsets)
    tgt_t, tgt_pinned = pinned_copy(csr.targets)
    ranks_host = None
    e2e_steps = max(3, min(args.steps, 10))

    def e2e_step():
        gg = G.GpuGraph.from_csr(off_pinned, tgt_pinned, dev)
        r = gg.pagerank_array(DAMPING, PR_ITERATIONS, 0.0)
        del gg
        return r["ranks"]

    e2e_step()
    d.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ranks_host = e2e_step()
    e2e_s = d.max(time.perf_counter() - t0)
    e2e_value = d.sum(float(B) * PR_ITERATIONS * e2e_steps) / e2e_s / 1e9
    assert ranks_host is not None and ranks_host.shape == (V,)
    del off_t, tgt_t

    line = {
        "metric": "PageRank iteration GB/s (algorithmic bytes 4E+12V+4 per iteration)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": d.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (f64 residual and dangling mass)",
        "data": "synthetic R-MAT (stands in for Graph500/GraphChallenge inputs)",
        "config": {
            "workload": f"R-MAT scale {args.scale}, edge factor {EDGE_FACTOR}, a=0.57 b=0.19 c=0.19, seed {SEED}; "
                        f"PageRank {PR_ITERATIONS} iterations, damping {DAMPING}, per step",
            "vertices": V,
            "csr_entries": E,
            "bytes_per_iteration": B,
            "l2": "inputs larger than L2 (CSR %.2f GB > 126 MB)" % ((4 * (V + 1) + 4 * E) / 1e9),
            "parallelism": f"replicas x{d.world}",
            "graph_generation_s": round(gen_s, 2),
        },
        "gpu_launches": int(launches),
        "roofline": roofline,
        "e2e": {
            "value": round(e2e_value, 2),
            "unit": "GB/s",
            "h2d_bytes_per_step": 4 * (V + 1) + 4 * E,
            "d2h_bytes_per_step": 4 * V,
            "what": "GpuGraph.from_csr(pinned host CSR) + pagerank(ranks to host), wall time",
        },
        "clocks": clk,
        "kernel_ms_per_step": {k: round(v[1], 4) for k, v in stats.items()},
    }

    if d.rank == 0 and d.world == 1:
        line["cpu_baseline"] = cpu_pagerank_sample(csr, B, seconds=10.0)
    if not args.no_secondary and d.world == 1:
        line["algorithms"] = secondary(csr, g, dev, args)
    return line


def cpu_pagerank_sample(csr, B: int, seconds: float) -> dict:
    """Oracle PageRank on the host cores: batches of iterations until ~`seconds`."""
    from oracle import oracle as O

    iterations, s = 0, 0.0
    batch = 2
    while s < seconds and iterations < 2000:
        t = time.perf_counter()
        O.pagerank(csr.offsets, csr.targets, DAMPING, batch, 0.0)
        s += time.perf_counter() - t
        iterations += batch
        batch = min(batch * 2, 64)
    return {
        "value": round(B * iterations / s / 1e9, 3),
        "unit": "GB/s",
        "cores": O.num_threads(),
        "kind": "port",
        "sample": f"{iterations} FP64 PageRank iterations of the oracle on the same graph ({s:.1f} s)",
    }


def secondary(csr, g, dev, args, k_truss: bool = True) -> dict:
    """BFS, triangle counting and k-truss on the resident graph (device time)."""
    out = {}
    V, E = csr.num_nodes, csr.num_edges
    m = E // 2
    sources = bfs_sources(csr, BFS_SOURCES, SEED)
    comp_edges = []
    for s in sources:
        r = g.bfs_array(int(s))
        comp_edges.append(component_edges(csr, r["distances"]))
    total_m = float(sum(comp_edges))
    for s in sources[:3]:
        g.bfs_array(int(s), copy_result=False)
    dev.timer_start()
    for s in sources:
        g.bfs_array(int(s), copy_result=False)
    bfs_ms = dev.timer_stop()
    bfs_bytes = sum(8 * c + 8 * V for c in comp_edges)
    out["bfs"] = {
        "metric": "BFS GTEPS (Graph500: component edges / time, 64 sources)",
        "value": round(total_m / (bfs_ms / 1e3) / 1e9, 3),
        "unit": "GTEPS",
        "ms_per_source": round(bfs_ms / len(sources), 4),
        "hbm_frac_of_measured": round(bfs_bytes / (bfs_ms / 1e3) / 1e9 / measured_peak()[0], 4),
    }
    g.triangle_count()
    dev.timer_start()
    reps = 2
    for _ in range(reps):
        tc = g.triangle_count()
    tc_ms = dev.timer_stop() / reps
    out["triangle_count"] = {
        "metric": "triangle counting edges/s (undirected edges / time)",
        "value": round(m / (tc_ms / 1e3), 1),
        "unit": "edges/s",
        "ms": round(tc_ms, 3),
        "triangles": tc["total_triangles"],
    }
    # The same BFS and triangle count with the learned schedule installed
    # (the shipped network), against the fixed rules measured above.
    from grafeo_cuda import schedule as sched

    if os.path.exists(sched.DEFAULT_WEIGHTS):
        ref_dist = g.bfs_array(int(sources[0]))["distances"]
        sched.install(dev)
        try:
            same = bool(np.array_equal(g.bfs_array(int(sources[0]))["distances"], ref_dist))
            for s in sources[:3]:
                g.bfs_array(int(s), copy_result=False)
            dev.timer_start()
            for s in sources:
                g.bfs_array(int(s), copy_result=False)
            lbfs_ms = dev.timer_stop()
            tc_l = g.triangle_count()
            dev.timer_start()
            for _ in range(reps):
                tc_l = g.triangle_count()
            ltc_ms = dev.timer_stop() / reps
        finally:
            dev.set_schedule(None)
        out["learned_schedule"] = {
            "bfs_gteps": round(total_m / (lbfs_ms / 1e3) / 1e9, 3),
            "bfs_speedup_vs_alpha_beta": round(bfs_ms / lbfs_ms, 3),
            "triangle_count_ms": round(ltc_ms, 3),
            "triangle_speedup_vs_fixed_buckets": round(tc_ms / ltc_ms, 3),
            "results_identical": same and tc_l["total_triangles"] == tc["total_triangles"],
        }
    if not k_truss:
        return out
    kt = {}
    dev.timer_start()
    for k in range(3, 9):
        r = g.k_truss_array(k)
        kt[k] = {"edges": int(len(r["edges"])), "rounds": r["iterations"]}
    kt_ms = dev.timer_stop()
    out["k_truss"] = {
        "metric": "k-truss edges/s (undirected edges / time, k = 3..8 sweep)",
        "value": round(6 * m / (kt_ms / 1e3), 1),
        "unit": "edges/s",
        "ms_total": round(kt_ms, 2),
        "per_k": kt,
    }
    return out


# ---------------------------------------------------------------- suite (configurations at scale)


def pagerank_gbs(g, dev, V: int, E: int, iterations: int = PR_ITERATIONS) -> dict:
    g.pagerank_array(DAMPING, iterations, 0.0, copy_result=False)
    dev.timer_start()
    g.pagerank_array(DAMPING, iterations, 0.0, copy_result=False)
    ms = dev.timer_stop()
    return {"metric": "PageRank iteration GB/s (4E+12V+4 bytes per iteration)",
            "value": round(pr_bytes(V, E) * iterations / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "ms_per_iteration": round(ms / iterations, 4)}


def directed_dangling_copy(csr, fraction: float, seed: int):
    """The directed copy of a symmetric CSR in which a seeded uniform
    `fraction` of the vertices lose their out-edges (they become dangling)."""
    V = csr.num_nodes
    rng = np.random.default_rng(seed)
    drop = np.zeros(V, dtype=bool)
    drop[rng.choice(V, size=int(round(fraction * V)), replace=False)] = True
    deg = np.diff(csr.offsets).astype(np.int64)
    keep_rows = ~drop
    offsets = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(np.where(keep_rows, deg, 0), out=offsets[1:])
    targets = csr.targets[np.repeat(keep_rows, deg)]
    return offsets.astype(np.uint32), targets, int(drop.sum())


def run_suite(args) -> dict:
    import grafeo_cuda as G
    from oracle import oracle as O

    dev = G.GpuDevice(0)
    out = {"suite": "four algorithms at scale; learned schedule against the fixed rules", "device": dev.name}
    graphs = (
        ("rmat22", "R-MAT scale 22, edge factor 16, a=0.57 b=0.19 c=0.19, seed 2",
         lambda: G.GpuGraph.generate_rmat(dev, 22, EDGE_FACTOR, *RMAT_ABC, seed=2)),
        ("er22", "Erdos-Renyi G(n = 4,194,304, 16n pairs -> average degree ~32), seed 3",
         lambda: G.GpuGraph.generate_erdos_renyi(dev, 1 << 22, 16 << 22, seed=3)),
    )
    for name, what, make in graphs:
        g = make()
        csr = g.to_csr()
        block = {"graph": what, "vertices": csr.num_nodes, "csr_entries": csr.num_edges,
                 "pagerank": pagerank_gbs(g, dev, csr.num_nodes, csr.num_edges)}
        block.update(secondary(csr, g, dev, args))
        out[name] = block
        del g
    # R-MAT 24, seed 5.
    t0 = time.time()
    g = G.GpuGraph.generate_rmat(dev, 24, EDGE_FACTOR, *RMAT_ABC, seed=5)
    dev.synchronize()
    gen_s = time.time() - t0
    csr = g.to_csr()
    V, E = csr.num_nodes, csr.num_edges
    s24 = {"graph": "R-MAT scale 24, edge factor 16, a=0.57 b=0.19 c=0.19, seed 5", "vertices": V,
           "csr_entries": E, "device_generation_s": round(gen_s, 3)}
    # Directed copy with 3 % dangling vertices: PageRank to tol 1e-7 (<= 100 iterations).
    doff, dtgt, ndrop = directed_dangling_copy(csr, 0.03, seed=5)
    gd = G.GpuGraph.from_csr(doff, dtgt, dev)
    gd.pagerank_directed(DAMPING, 2, 0.0)  # builds the transpose plan (not timed)
    dev.timer_start()
    pr = gd.pagerank_directed(DAMPING, 100, 1e-7)
    pr_ms = dev.timer_stop()
    t0 = time.perf_counter()
    ref = O.pagerank_directed(doff, dtgt, DAMPING, pr["iterations"], 0.0)
    ref_s = time.perf_counter() - t0
    err = np.asarray(pr["ranks"], dtype=np.float64) - ref["ranks"]
    s24["pagerank_directed"] = {
        "dangling_vertices": ndrop, "csr_entries": int(len(dtgt)), "damping": DAMPING, "tolerance": 1e-7,
        "iterations": pr["iterations"], "converged": pr["converged"], "device_ms": round(pr_ms, 2),
        "ms_per_iteration": round(pr_ms / max(pr["iterations"], 1), 4),
        "l1_error_vs_fp64_oracle": float(np.abs(err).sum()), "linf_error_vs_fp64_oracle": float(np.abs(err).max()),
        "oracle": f"FP64 power iteration, same {pr['iterations']} iterations, {O.num_threads()} threads, {ref_s:.1f} s",
    }
    del gd
    # Truss decomposition (every k up to the maximum trussness).
    dev.timer_start()
    td = g.truss_decomposition(copy_result=False)
    td_ms = dev.timer_stop()
    s24["truss_decomposition"] = {"max_trussness": td["max_trussness"], "rounds": td["rounds"],
                                  "device_ms": round(td_ms, 1),
                                  "edges_per_s": round((E // 2) / (td_ms / 1e3), 1)}
    # BFS and triangles, with the learned schedule against the fixed rules.
    s24.update(secondary(csr, g, dev, args, k_truss=False))
    out["rmat24"] = s24
    return out


# ---------------------------------------------------------------- reference arm (CPU)


def run_reference(args, d: Dist) -> dict | None:
    if d.rank != 0:
        return None
    from oracle import oracle as O

    csr, gen_s = make_graph(args.scale)
    V, E = csr.num_nodes, csr.num_edges
    B = pr_bytes(V, E)
    sample_iters = PR_ITERATIONS  # the same 50-iteration step as the GPU arm
    for _ in range(max(args.warmup, 1)):
        O.pagerank(csr.offsets, csr.targets, DAMPING, sample_iters, 0.0)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.pagerank(csr.offsets, csr.targets, DAMPING, sample_iters, 0.0)
    s = time.perf_counter() - t
    value = B * sample_iters * args.steps / s / 1e9
    sample = f"{sample_iters} FP64 PageRank iterations per step on the full graph"
    return {
        "impl": "reference",
        "metric": "PageRank iteration GB/s (algorithmic bytes 4E+12V+4 per iteration)",
        "value": round(value, 3),
        "unit": "GB/s",
        "n_gpus": d.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(s / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic R-MAT (stands in for Graph500/GraphChallenge inputs)",
        "config": {
            "workload": f"R-MAT scale {args.scale}, edge factor {EDGE_FACTOR}, a=0.57 b=0.19 c=0.19, seed {SEED}; "
                        f"PageRank damping {DAMPING}",
            "vertices": V,
            "csr_entries": E,
        },
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Grafeo 0.6.3's Rust CPU algorithms cannot be built here (no Rust toolchain, crate not vendored); "
                "the oracle's OpenMP restatement of the same algorithm stands in for them",
    }


def run_bfs_breakdown() -> dict:
    """Device time of 16 searches (CUDA events around the run) against the sum
    of their kernels' own event times, and the per-kernel split."""
    import grafeo_cuda as G

    dev = G.GpuDevice(0)
    out = {"bfs_breakdown": "16 random sources per graph; ms per search", "device": dev.name}
    graphs = (
        ("rmat22", lambda: G.GpuGraph.generate_rmat(dev, 22, EDGE_FACTOR, *RMAT_ABC, seed=2)),
        ("er22", lambda: G.GpuGraph.generate_erdos_renyi(dev, 1 << 22, 16 << 22, seed=3)),
    )
    for name, make in graphs:
        g = make()
        sources = [int(x) for x in np.random.default_rng(1).integers(0, g.num_nodes, 16)]
        for s in sources[:3]:
            g.bfs_array(s, copy_result=False)
        dev.timer_start()
        for s in sources:
            g.bfs_array(s, copy_result=False)
        wall_ms = dev.timer_stop()
        dev.set_kernel_timing(True)
        dev.reset_stats()
        depth = 0
        for s in sources:
            depth += g.bfs_array(s, copy_result=False)["max_depth"]
        stats = dev.kernel_stats()
        dev.set_kernel_timing(False)
        kernel_ms = sum(v[1] for v in stats.values())
        out[name] = {
            "ms_per_search": round(wall_ms / len(sources), 4),
            "kernel_ms_per_search": round(kernel_ms / len(sources), 4),
            "kernel_share": round(kernel_ms / wall_ms, 3) if wall_ms else None,
            "levels_per_search": depth / len(sources),
            "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)}
                        for k, v in sorted(stats.items(), key=lambda kv: -kv[1][1])},
        }
        del g
    return out


def main():
    args = parse_args()
    if args.suite:
        print(json.dumps(run_suite(args)), flush=True)
        return
    if args.bfs_breakdown:
        print(json.dumps(run_bfs_breakdown()), flush=True)
        return
    d = Dist()
    try:
        line = run_reference(args, d) if args.impl == "reference" else run_ours(args, d)
        if d.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        d.close()


if __name__ == "__main__":
    main()
