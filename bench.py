#!/usr/bin/env python
"""Benchmark of the four graph hot paths; headline on R-MAT scale 24 (seed 5).

Headline (`metric`/`value`): PageRank iteration throughput in GB/s of
algorithmic traffic, B = 4E + 12V + 4 bytes per iteration (offsets and
targets of the pulled in-CSR, one read of the contribution vector and one
write of the ranks), on the large skewed configuration: R-MAT scale 24
(16,777,216 vertices, edge factor 16, a=0.57 b=0.19 c=0.19, seed 5),
symmetrised and deduplicated, then a directed copy in which a seeded
uniform 3 % of the vertices lose their out-edges (dangling). One step is one
PageRank run at damping 0.85 to an L1 change below 1e-7 (at most 100
iterations): FP32 row sums with compensation, FP64 residual and dangling
mass. Its L1 and Linf error against the FP64 oracle at the same iteration
count ride along (computed outside the timed region).

  value  device time (CUDA events on the library's stream) with the CSR
         already resident in HBM (2 GB, larger than L2); the transpose plan
         is built once per graph, before the timed region.
  e2e    the same metric through the public API with host buffers: every step
         copies the directed CSR from pinned host memory (GpuGraph.from_csr,
         which validates it), builds the transpose plan, runs PageRank and
         copies the ranks back; wall time.
  roofline  the dominant kernel (one launch = one iteration) against the
         measured HBM copy bandwidth.
  cpu_baseline  the oracle's OpenMP FP64 PageRank on this host's cores: the
         same iteration count on the same graph (the run the error is taken
         from).
  harness  one record per algorithm and graph in the reference's
         GpuBenchmarkResult layout (crates/grafeo-cuda-algos/src/harness.rs:14-52),
         with every run's kernel time, the median and the best.
  algorithms  BFS (64 seeded non-isolated sources), triangle counting and the
         truss decomposition on the symmetric R-MAT 24 graph, with the learned
         schedule against the fixed rules; PageRank, BFS, triangles and the
         k-truss sweep k = 3..8 on R-MAT 22 (seed 2) and Erdos-Renyi 2^22
         (seed 3).

`--impl reference` times the reference's CPU implementation of the path (the
oracle port; Grafeo's own Rust crate cannot be built here) on the same metric
and configuration; its graph comes from the oracle's own generator, so it
loads nothing of this project's library.

Multi-GPU (torchrun): one process per GPU, each a full replica of the graph
running its own PageRank (no data-path collective; weak scaling); value is the
work of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import socket
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grafeo-cuda_b200"))
sys.path.insert(0, ROOT)

EDGE_FACTOR = 16
RMAT_ABC = (0.57, 0.19, 0.19)
DAMPING = 0.85
# The headline configuration: R-MAT 24, seed 5, directed copy with 3 % dangling vertices.
SCALE, SEED = 24, 5
DANGLING = 0.03
TOLERANCE = 1e-7
MAX_ITERATIONS = 100
# The secondary configurations (R-MAT 22 seed 2, Erdos-Renyi 2^22 seed 3).
PR_ITERATIONS = 50
BFS_SOURCES = 64
RUNS = 5
METRIC = "PageRank iteration GB/s (algorithmic bytes 4E+12V+4 per iteration, E = pulled in-CSR entries)"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--no-secondary", action="store_true", help="skip the algorithms block and the harness records")
    ap.add_argument("--save", metavar="DIR", help="also write every harness record to DIR/gpu_<algorithm>_<dataset>.json")
    ap.add_argument("--bfs-breakdown", action="store_true",
                    help="instead of the headline: BFS from 16 random sources on R-MAT 22, Erdos-Renyi 2^22 and "
                         "R-MAT 24, device time per search with the level loop on the device and on the host, "
                         "against the sum of its kernels' CUDA-event times, per kernel; one JSON document")
    ap.add_argument("--pr-ceiling", action="store_true",
                    help="instead of the headline: PageRank's row kernel per iteration against the gather probe "
                         "(its plan's target stream and contribution gathers alone) on R-MAT 22, Erdos-Renyi 2^22 "
                         "and the R-MAT 24 directed copy; one JSON document")
    ap.add_argument("--transpose-breakdown", action="store_true",
                    help="instead of the headline: the directed PageRank plan build (device transpose by radix sort, "
                         "degree-class relabelling) of the R-MAT directed copy at --scale (24: seed 5, 22: seed 2), "
                         "device ms per kernel, median of 4 builds; one JSON document")
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
    """DRAM bytes per iteration recorded by the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_iteration_full_size:"):
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
                 "-lms", "100"],
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


def pinned_copy(arr: np.ndarray):
    """Copies a u32 array into page-locked host memory (torch pin_memory)."""
    import torch

    t = torch.empty(arr.size, dtype=torch.int32, pin_memory=torch.cuda.is_available())
    view = t.numpy().view(np.uint32)
    view[:] = arr
    return t, view


def bfs_sources(offsets: np.ndarray, count: int, seed: int) -> np.ndarray:
    deg = np.diff(offsets)
    rng = np.random.default_rng(seed)
    return rng.choice(np.flatnonzero(deg > 0), size=count, replace=False)


def component_edges(offsets: np.ndarray, dist: np.ndarray) -> int:
    """Undirected edges with both ends in the reached component (Graph500 m)."""
    deg = np.diff(offsets).astype(np.int64)
    return int(deg[dist >= 0].sum() // 2)


def directed_dangling_copy(offsets: np.ndarray, targets: np.ndarray, fraction: float, seed: int):
    """The directed copy of a symmetric CSR in which a seeded uniform
    `fraction` of the vertices lose their out-edges (they become dangling)."""
    V = len(offsets) - 1
    rng = np.random.default_rng(seed)
    drop = np.zeros(V, dtype=bool)
    drop[rng.choice(V, size=int(round(fraction * V)), replace=False)] = True
    deg = np.diff(offsets).astype(np.int64)
    kept = np.where(drop, 0, deg)
    new_offsets = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(kept, out=new_offsets[1:])
    new_targets = targets[np.repeat(~drop, deg)]
    return new_offsets.astype(np.uint32), new_targets, int(drop.sum())


def workload_config(scale: int, V: int, E_pull: int, n_dangling: int, world: int) -> dict:
    """The headline's `config`, identical in both arms."""
    return {
        "workload": f"R-MAT scale {scale}, edge factor {EDGE_FACTOR}, a=0.57 b=0.19 c=0.19, seed {SEED}, "
                    f"symmetrised and deduplicated; directed copy with {DANGLING:.0%} of the vertices dangling "
                    f"(seeded); PageRank damping {DAMPING} until the L1 change is below {TOLERANCE:g} "
                    f"(at most {MAX_ITERATIONS} iterations); throughput per iteration",
        "vertices": V,
        "csr_entries": E_pull,
        "dangling_vertices": n_dangling,
        "bytes_per_iteration": pr_bytes(V, E_pull),
        "l2": ("inputs larger than L2 (in-CSR %.2f GB > 126 MB)" if 4 * (V + 1) + 4 * E_pull > 126e6
               else "inputs smaller than L2 (in-CSR %.2f GB)") % ((4 * (V + 1) + 4 * E_pull) / 1e9),
        "parallelism": f"replicas x{world}",
    }


def stats(runs_ms: list[float]) -> dict:
    return {"median_ms": round(statistics.median(runs_ms), 4), "best_ms": round(min(runs_ms), 4),
            "runs_ms": [round(x, 4) for x in runs_ms]}


def platform_info(gpu: str) -> str:
    """The reference's platform string (harness.rs:162-170)."""
    return f"{platform.system().lower()} / {platform.machine()} / {socket.gethostname()} / GPU: {gpu}"


def harness_record(dataset: str, algorithm: str, V: int, E: int, transfer_s: float, runs_ms: list[float],
                   teps_edges: float, gpu: str, extra: dict) -> dict:
    """One GpuBenchmarkResult (harness.rs:14-52): best kernel time over the
    runs, transfer = CSR upload with validation, teps = edges / best."""
    best = min(runs_ms) / 1e3
    return {
        "dataset": dataset, "algorithm": algorithm, "vertices": V, "edges": E,
        "time_s": transfer_s + best, "transfer_time_s": transfer_s, "kernel_time_s": best,
        "teps": teps_edges / best if best > 0 else 0.0,
        "runs": [x / 1e3 for x in runs_ms],
        "platform": platform_info(gpu), "gpu_device": gpu,
        "extra": dict(extra, median_kernel_time_s=statistics.median(runs_ms) / 1e3),
    }


def timed(dev, fn, runs: int = RUNS) -> tuple[list[float], object]:
    """Device time of `runs` calls (CUDA events around each), after one warm-up call."""
    out = fn()
    times = []
    for _ in range(runs):
        dev.timer_start()
        out = fn()
        times.append(dev.timer_stop())
    return times, out


# ---------------------------------------------------------------- our implementation


def run_ours(args, d: Dist) -> dict | None:
    import grafeo_cuda as G

    dev = G.GpuDevice(d.local_rank)
    t0 = time.perf_counter()
    g = G.GpuGraph.generate_rmat(dev, args.scale, EDGE_FACTOR, *RMAT_ABC, seed=SEED)
    sym = g.to_csr()
    doff, dtgt, ndrop = directed_dangling_copy(sym.offsets, sym.targets, DANGLING, SEED)
    prep_s = time.perf_counter() - t0
    V, E = len(doff) - 1, len(dtgt)
    B = pr_bytes(V, E)
    t0 = time.perf_counter()
    gd = G.GpuGraph.from_csr(doff, dtgt, dev)
    dev.synchronize()
    transfer_s = time.perf_counter() - t0
    gd.pagerank_directed(DAMPING, 2, 0.0, copy_result=False)  # builds the transpose plan

    iters = []

    def pr_step():
        r = gd.pagerank_directed(DAMPING, MAX_ITERATIONS, TOLERANCE, copy_result=False)
        iters.append(r["iterations"])

    # -- value: CSR resident in HBM, device time over K steps, max over ranks
    for _ in range(args.warmup):
        pr_step()
    dev.synchronize()
    iters.clear()
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
    total_bytes = d.sum(float(B) * sum(iters))
    value = total_bytes / (ms_max / 1e3) / 1e9
    step_iterations = iters[-1]

    # -- roofline of the dominant kernel: per-launch device time with events
    dev.set_kernel_timing(True)
    dev.reset_stats()
    pr_step()
    kstats = dev.kernel_stats()
    dev.set_kernel_timing(False)
    # The SpMV of one iteration (B bytes) is two kernels: pr_rows (segments of
    # the rows of >= 1024 entries, and the rows without entries) and pr_chunks
    # (the other rows, as a stream of 256-entry chunks). Iterations are queued
    # in chunks and the launches queued past convergence return at once, so the
    # time per iteration is the kernels' total time over the iterations run,
    # not over their launches.
    spmv = [k for k in ("pr_rows", "pr_chunks") if k in kstats]
    kernel = "+".join(spmv)
    tile_n = kstats[spmv[0]][0]
    tile_ms = sum(kstats[k][1] for k in spmv)
    step_ms = sum(v[1] for v in kstats.values())
    per_iteration_ms = tile_ms / max(step_iterations, 1)
    peak, peak_kind = measured_peak()
    achieved = B / (per_iteration_ms / 1e3) / 1e9
    roofline = {
        "kernel": kernel,
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": peak,
        "peak_kind": peak_kind,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "frac_of_8tbs_spec": round(achieved / 8000.0, 4),
        "traffic": profiled_traffic(f"pagerank_spmv_rmat{args.scale}_directed.md"),
        "traffic_is": "dram__bytes_read.sum + dram__bytes_write.sum of both kernels per iteration (ncu)",
        "algorithmic_bytes_per_launch": B,
        "ms_per_working_launch": round(per_iteration_ms, 5),
        "kernel_ms_per_step": {k: round(kstats[k][1], 4) for k in spmv},
        "launches_per_step": tile_n,
        "working_launches_per_step": step_iterations,
        "share_of_step": round(tile_ms / step_ms, 4) if step_ms else None,
    }

    # -- the result, for the error against the FP64 oracle (not timed)
    result = gd.pagerank_directed(DAMPING, MAX_ITERATIONS, TOLERANCE)
    assert result["iterations"] == step_iterations

    # -- e2e through the public API with host buffers
    off_t, off_pinned = pinned_copy(doff)
    tgt_t, tgt_pinned = pinned_copy(dtgt)
    e2e_steps = max(3, min(args.steps, 8))
    e2e_iters = []

    def e2e_step():
        gg = G.GpuGraph.from_csr(off_pinned, tgt_pinned, dev)
        r = gg.pagerank_directed(DAMPING, MAX_ITERATIONS, TOLERANCE)
        del gg
        e2e_iters.append(r["iterations"])
        return r["ranks"]

    # Untimed warm-up steps, as many as the headline's (at least 3): with the
    # headline's graphs resident, the first steps of a process grow the
    # stream-ordered pool and run 30-40 ms slower than the steady state.
    for _ in range(max(args.warmup, 3)):
        e2e_step()
    e2e_iters.clear()
    d.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ranks_host = e2e_step()
    e2e_s = d.max(time.perf_counter() - t0)
    e2e_value = d.sum(float(B) * sum(e2e_iters)) / e2e_s / 1e9
    assert ranks_host.shape == (V,)
    # One more step, outside the timed loop, with per-kernel timing on: where
    # an e2e step's time goes (wall time of the two calls, device time per kernel).
    dev.set_kernel_timing(True)
    dev.reset_stats()
    t_a = time.perf_counter()
    gg = G.GpuGraph.from_csr(off_pinned, tgt_pinned, dev)
    dev.synchronize()
    t_b = time.perf_counter()
    gg.pagerank_directed(DAMPING, MAX_ITERATIONS, TOLERANCE)
    t_c = time.perf_counter()
    del gg
    dev.synchronize()
    t_d = time.perf_counter()
    e2e_kernels = dev.kernel_stats()
    dev.set_kernel_timing(False)
    e2e_breakdown = {
        "from_csr_ms": round((t_b - t_a) * 1e3, 2),
        "pagerank_directed_ms": round((t_c - t_b) * 1e3, 2),
        "graph_release_ms": round((t_d - t_c) * 1e3, 2),
        "kernel_ms": {k: round(v[1], 3) for k, v in sorted(e2e_kernels.items(), key=lambda kv: -kv[1][1])[:12]},
        "note": "one extra step with per-kernel CUDA events on (slightly slower than the timed steps)",
    }
    del off_t, tgt_t

    line = {
        "metric": METRIC,
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
        "config": workload_config(args.scale, V, E, ndrop, d.world),
        "iterations_per_step": step_iterations,
        "converged": result["converged"],
        "graph_preparation_s": round(prep_s, 2),
        "gpu_launches": int(launches),
        "roofline": roofline,
        "e2e": {
            "value": round(e2e_value, 2),
            "unit": "GB/s",
            "h2d_bytes_per_step": 4 * (V + 1) + 4 * E,
            "d2h_bytes_per_step": 4 * V,
            "what": "GpuGraph.from_csr(pinned host CSR) + pagerank_directed(ranks to host), wall time; "
                    "every step uploads, validates, transposes and plans the graph",
            "ms_per_step": round(e2e_s / e2e_steps * 1e3, 2),
            "breakdown": e2e_breakdown,
        },
        "clocks": clk,
        "kernel_ms_per_step": {k: round(v[1], 4) for k, v in kstats.items()},
    }

    if d.rank == 0 and d.world == 1:
        # The FP64 oracle at the same iteration count, timed: the CPU baseline and the error.
        from oracle import oracle as O

        to, tt = O.transpose_sorted(doff, dtgt)
        t0 = time.perf_counter()
        ref = O.pagerank(to, tt, DAMPING, step_iterations, 0.0, out_degree=np.diff(doff))
        ref_s = time.perf_counter() - t0
        err = result["ranks"].astype(np.float64) - ref["ranks"]
        line["accuracy"] = {
            "l1_error_vs_fp64_oracle": float(np.abs(err).sum()),
            "linf_error_vs_fp64_oracle": float(np.abs(err).max()),
            "oracle": f"FP64 power iteration over the same in-CSR, {step_iterations} iterations",
            "target_l1": 1e-6,
        }
        line["cpu_baseline"] = {
            "value": round(B * step_iterations / ref_s / 1e9, 3),
            "unit": "GB/s",
            "cores": O.num_threads(),
            "kind": "port",
            "sample": f"the oracle's FP64 PageRank, {step_iterations} iterations on the same in-CSR "
                      f"({ref_s:.1f} s; the run the error above is taken from)",
        }
        del to, tt
    if not args.no_secondary and d.world == 1:
        harness = []
        # Headline record: kernel time of separate runs of the same step.
        pr_runs, _ = timed(dev, lambda: gd.pagerank_directed(DAMPING, MAX_ITERATIONS, TOLERANCE, copy_result=False))
        harness.append(harness_record(
            f"rmat{args.scale}_seed{SEED}_directed_dangling3", "gpu_pagerank_directed", V, E, transfer_s, pr_runs,
            float(E) * step_iterations, dev.name,
            {"iterations": step_iterations, "converged": result["converged"], "damping": DAMPING,
             "tolerance": TOLERANCE, "gbs_per_iteration_best": B * step_iterations / (min(pr_runs) / 1e3) / 1e9}))
        del gd
        algos = {}
        algos[f"rmat{args.scale}"] = symmetric_block(g, sym, dev, f"rmat{args.scale}_seed{SEED}", harness,
                                                     decomposition=True, sweep=False, pagerank=False)
        del g, sym
        for name, make in (
            ("rmat22", lambda: G.GpuGraph.generate_rmat(dev, 22, EDGE_FACTOR, *RMAT_ABC, seed=2)),
            ("er22", lambda: G.GpuGraph.generate_erdos_renyi(dev, 1 << 22, 16 << 22, seed=3)),
        ):
            gg = make()
            algos[name] = symmetric_block(gg, gg.to_csr(), dev, name + ("_seed2" if name == "rmat22" else "_seed3"),
                                          harness, decomposition=False, sweep=True, pagerank=True)
            del gg
        algos["rmat14"] = small_config_block(dev, harness)
        line["algorithms"] = algos
        line["harness"] = harness
        if args.save:
            os.makedirs(args.save, exist_ok=True)
            for rec in harness:
                with open(os.path.join(args.save, f"gpu_{rec['algorithm']}_{rec['dataset']}.json"), "w") as f:
                    json.dump(rec, f, indent=2)
    return line


def symmetric_block(g, csr, dev, dataset: str, harness: list, decomposition: bool, sweep: bool,
                    pagerank: bool) -> dict:
    """BFS, triangles (with the learned schedule against the fixed rules),
    and PageRank, the k-truss sweep or the truss decomposition, on a
    resident symmetric graph; device times, RUNS runs each."""
    import grafeo_cuda as G
    from grafeo_cuda import schedule as sched

    out = {"vertices": csr.num_nodes, "csr_entries": csr.num_edges}
    V, E = csr.num_nodes, csr.num_edges
    m = E // 2
    peak = measured_peak()[0]
    t0 = time.perf_counter()
    G.GpuGraph.from_csr_arrays(csr, dev)  # upload + validation time, the harness transfer figure
    dev.synchronize()
    transfer_s = time.perf_counter() - t0
    if pagerank:
        runs, _ = timed(dev, lambda: g.pagerank_array(DAMPING, PR_ITERATIONS, 0.0, copy_result=False))
        B = pr_bytes(V, E)
        out["pagerank"] = {"metric": "PageRank iteration GB/s (4E+12V+4 bytes per iteration), 50 iterations",
                           "value": round(B * PR_ITERATIONS / (statistics.median(runs) / 1e3) / 1e9, 2),
                           "unit": "GB/s", "hbm_frac_of_measured": round(
                               B * PR_ITERATIONS / (statistics.median(runs) / 1e3) / 1e9 / peak, 4),
                           "ms_per_iteration_median": round(statistics.median(runs) / PR_ITERATIONS, 4),
                           **stats(runs)}
        harness.append(harness_record(dataset, "gpu_pagerank", V, E, transfer_s, runs, float(E) * PR_ITERATIONS,
                                      dev.name, {"iterations": PR_ITERATIONS, "damping": DAMPING}))
    # BFS from 64 seeded non-isolated sources, RUNS runs each.
    sources = bfs_sources(csr.offsets, BFS_SOURCES, 2)
    comp, per_source_best, teps = [], [], []
    total_median = 0.0
    for s in sources:
        r = g.bfs_array(int(s))
        comp.append(component_edges(csr.offsets, r["distances"]))
        runs, _ = timed(dev, lambda: g.bfs_array(int(s), copy_result=False))
        per_source_best.append(min(runs))
        total_median += statistics.median(runs)
        teps.append(E / (min(runs) / 1e3))
    m_cc = float(sum(comp))
    bfs_bytes = sum(8 * c + 8 * V for c in comp)
    out["bfs"] = {
        "metric": "BFS GTEPS (Graph500: component edges over time; 64 sources, median of 5 runs each)",
        "value": round(m_cc / (total_median / 1e3) / 1e9, 3), "unit": "GTEPS",
        "ms_per_source_median": round(total_median / len(sources), 4),
        "hbm_frac_of_measured": round(bfs_bytes / (total_median / 1e3) / 1e9 / peak, 4),
        "reference_teps_harmonic_mean": round(len(teps) / sum(1.0 / t for t in teps), 1),
    }
    harness.append(harness_record(dataset, "gpu_bfs", V, E, transfer_s, per_source_best, float(E), dev.name,
                                  {"sources": len(sources), "runs_are": "best of 5 per source",
                                   "teps_harmonic_mean": out["bfs"]["reference_teps_harmonic_mean"]}))
    runs, tc = timed(dev, g.triangle_count)
    out["triangle_count"] = {"metric": "triangle counting edges/s (undirected edges / time)",
                             "value": round(m / (statistics.median(runs) / 1e3), 1), "unit": "edges/s",
                             "triangles": tc["total_triangles"], **stats(runs)}
    harness.append(harness_record(dataset, "gpu_triangle_count", V, E, transfer_s, runs, float(E), dev.name,
                                  {"triangles": tc["total_triangles"]}))
    # The same BFS and triangle count with the learned schedule (the shipped network).
    if os.path.exists(sched.DEFAULT_WEIGHTS):
        ref_dist = g.bfs_array(int(sources[0]))["distances"]
        sched.install(dev)
        try:
            same = bool(np.array_equal(g.bfs_array(int(sources[0]))["distances"], ref_dist))
            lmed = 0.0
            for s in sources:
                runs_l, _ = timed(dev, lambda: g.bfs_array(int(s), copy_result=False))
                lmed += statistics.median(runs_l)
            runs_t, tc_l = timed(dev, g.triangle_count)
        finally:
            dev.set_schedule(None)
        out["learned_schedule"] = {
            "bfs_gteps": round(m_cc / (lmed / 1e3) / 1e9, 3),
            "bfs_speedup_vs_alpha_beta": round(total_median / lmed, 3),
            "triangle_count_ms_median": round(statistics.median(runs_t), 3),
            "triangle_speedup_vs_fixed_buckets": round(out["triangle_count"]["median_ms"] / statistics.median(runs_t), 3),
            "results_identical": same and tc_l["total_triangles"] == tc["total_triangles"],
        }
    if sweep:
        per_k = {}

        def sweep_once():
            for k in range(3, 9):
                r = g.k_truss_array(k)
                per_k[k] = {"edges": int(len(r["edges"])), "rounds": r["iterations"]}

        runs, _ = timed(dev, sweep_once)
        out["k_truss"] = {"metric": "k-truss edges/s (undirected edges / time, k = 3..8 sweep)",
                          "value": round(6 * m / (statistics.median(runs) / 1e3), 1), "unit": "edges/s",
                          "per_k": per_k, **stats(runs)}
        harness.append(harness_record(dataset, "gpu_ktruss_sweep_3_8", V, E, transfer_s, runs, 6.0 * E, dev.name,
                                      {"per_k": per_k}))
    if decomposition:
        runs, td = timed(dev, lambda: g.truss_decomposition(copy_result=False), runs=3)
        out["truss_decomposition"] = {"metric": "truss decomposition edges/s (undirected edges / time)",
                                      "value": round(m / (statistics.median(runs) / 1e3), 1), "unit": "edges/s",
                                      "max_trussness": td["max_trussness"], "rounds": td["rounds"], **stats(runs)}
        harness.append(harness_record(dataset, "gpu_truss_decomposition", V, E, transfer_s, runs, float(E), dev.name,
                                      {"max_trussness": td["max_trussness"], "rounds": td["rounds"]}))
    return out


def small_config_block(dev, harness: list) -> dict:
    """The plain method at small size: R-MAT 14 seed 1; PageRank 20
    iterations (tol 1e-6), BFS from vertex 0, triangles, k-truss k = 4;
    device times, RUNS runs each."""
    import grafeo_cuda as G

    g = G.GpuGraph.generate_rmat(dev, 14, EDGE_FACTOR, *RMAT_ABC, seed=1)
    V, E = g.num_nodes, g.num_edges
    out = {"vertices": V, "csr_entries": E}
    runs, r = timed(dev, lambda: g.pagerank_array(DAMPING, 20, 1e-6, copy_result=False))
    out["pagerank"] = {"iterations": r["iterations"], "ms_median": round(statistics.median(runs), 4),
                       "gbs": round(pr_bytes(V, E) * r["iterations"] / (statistics.median(runs) / 1e3) / 1e9, 1)}
    harness.append(harness_record("rmat14_seed1", "gpu_pagerank", V, E, 0.0, runs, float(E) * r["iterations"],
                                  dev.name, {"iterations": r["iterations"]}))
    runs, r = timed(dev, lambda: g.bfs_array(0, copy_result=False))
    out["bfs_from_0"] = {"reachable": r["reachable"], "max_depth": r["max_depth"],
                         "ms_median": round(statistics.median(runs), 4)}
    harness.append(harness_record("rmat14_seed1", "gpu_bfs", V, E, 0.0, runs, float(E), dev.name,
                                  {"source_node": 0, "reachable_nodes": r["reachable"], "max_depth": r["max_depth"]}))
    runs, r = timed(dev, g.triangle_count)
    out["triangle_count"] = {"triangles": r["total_triangles"], "ms_median": round(statistics.median(runs), 4)}
    harness.append(harness_record("rmat14_seed1", "gpu_triangle_count", V, E, 0.0, runs, float(E), dev.name,
                                  {"triangles": r["total_triangles"]}))
    runs, r = timed(dev, lambda: g.k_truss_array(4))
    out["k_truss_4"] = {"edges": int(len(r["edges"])), "rounds": r["iterations"],
                        "ms_median": round(statistics.median(runs), 4)}
    harness.append(harness_record("rmat14_seed1", "gpu_ktruss", V, E, 0.0, runs, float(E), dev.name,
                                  {"k": 4, "truss_edges": int(len(r["edges"])), "iterations": r["iterations"]}))
    return out


# ---------------------------------------------------------------- reference arm (CPU)


def run_reference(args, d: Dist) -> dict | None:
    """The oracle's FP64 PageRank on the host cores: the graph from the
    oracle's own generator (equal to the library's, checked by the tests),
    the same directed copy and in-CSR; each step a bounded sample of
    iterations of the same workload."""
    if d.rank != 0:
        return None
    from oracle import oracle as O

    t0 = time.perf_counter()
    sym = O.generate_rmat(args.scale, EDGE_FACTOR, *RMAT_ABC, SEED)
    doff, dtgt, ndrop = directed_dangling_copy(sym.offsets, sym.targets, DANGLING, SEED)
    del sym
    to, tt = O.transpose_sorted(doff, dtgt)
    outdeg = np.diff(doff)
    prep_s = time.perf_counter() - t0
    V, E = len(doff) - 1, len(dtgt)
    B = pr_bytes(V, E)
    sample_iters = 2  # per step: a bounded sample of the run to tolerance
    for _ in range(max(args.warmup, 1)):
        O.pagerank(to, tt, DAMPING, sample_iters, 0.0, out_degree=outdeg)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.pagerank(to, tt, DAMPING, sample_iters, 0.0, out_degree=outdeg)
    s = time.perf_counter() - t
    value = B * sample_iters * args.steps / s / 1e9
    return {
        "impl": "reference",
        "metric": METRIC,
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
        "config": workload_config(args.scale, V, E, ndrop, d.world),
        "graph_preparation_s": round(prep_s, 2),
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
                         "sample": f"{sample_iters} FP64 PageRank iterations per step on the full in-CSR "
                                   f"(the GPU step runs the same iterations to tolerance)"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Grafeo 0.6.3's Rust CPU algorithms cannot be built here (no Rust toolchain, crate not vendored); "
                "the oracle's OpenMP restatement of the same algorithm stands in for them",
    }


def run_bfs_breakdown() -> dict:
    """Device time of 16 searches (CUDA events around the run) with the level
    loop on the device and driven from the host, against the sum of the
    kernels' own event times (host-driven, per-kernel timing on), and the
    per-kernel split."""
    import grafeo_cuda as G

    dev = G.GpuDevice(0)
    out = {"bfs_breakdown": "16 random sources per graph; ms per search", "device": dev.name}
    graphs = (
        ("rmat22", lambda: G.GpuGraph.generate_rmat(dev, 22, EDGE_FACTOR, *RMAT_ABC, seed=2)),
        ("er22", lambda: G.GpuGraph.generate_erdos_renyi(dev, 1 << 22, 16 << 22, seed=3)),
        ("rmat24", lambda: G.GpuGraph.generate_rmat(dev, 24, EDGE_FACTOR, *RMAT_ABC, seed=5)),
    )
    for name, make in graphs:
        g = make()
        sources = [int(x) for x in np.random.default_rng(1).integers(0, g.num_nodes, 16)]
        loop_ms = {}
        for on in (True, False):
            dev.set_bfs_device_loop(on)
            for s in sources[:3]:
                g.bfs_array(s, copy_result=False)
            dev.timer_start()
            for s in sources:
                g.bfs_array(s, copy_result=False)
            loop_ms[on] = dev.timer_stop()
        dev.set_bfs_device_loop(True)
        wall_ms = loop_ms[False]
        dev.set_kernel_timing(True)
        dev.reset_stats()
        depth = 0
        for s in sources:
            depth += g.bfs_array(s, copy_result=False)["max_depth"]
        kstats = dev.kernel_stats()
        dev.set_kernel_timing(False)
        kernel_ms = sum(v[1] for v in kstats.values())
        out[name] = {
            "ms_per_search_device_loop": round(loop_ms[True] / len(sources), 4),
            "ms_per_search": round(wall_ms / len(sources), 4),
            "kernel_ms_per_search": round(kernel_ms / len(sources), 4),
            "kernel_share": round(kernel_ms / wall_ms, 3) if wall_ms else None,
            "levels_per_search": depth / len(sources),
            "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)}
                        for k, v in sorted(kstats.items(), key=lambda kv: -kv[1][1])},
        }
        del g
    return out


def run_pr_ceiling() -> dict:
    """PageRank's row kernels against the floor of a pull SpMV on their plan:
    per graph, the device time per iteration of pr_rows + pr_chunks (per-kernel CUDA events, a
    fixed iteration count) and the gather probe's device time per pass (the
    plan's relabelled targets streamed and each contribution gathered, nothing
    else, same grid and CTA shape; median of 3 x 20 passes)."""
    import grafeo_cuda as G

    dev = G.GpuDevice(0)
    out = {"pr_ceiling": "pr_rows + pr_chunks ms per iteration against the gather probe's ms per pass on the same plan",
           "device": dev.name}
    for name in ("rmat22", "er22", "rmat24"):
        if name == "rmat24":
            g0 = G.GpuGraph.generate_rmat(dev, 24, EDGE_FACTOR, *RMAT_ABC, seed=5)
            csr = g0.to_csr()
            del g0
            off, tgt, _ = directed_dangling_copy(csr.offsets, csr.targets, 0.03, 5)
            del csr
            g = G.GpuGraph.from_csr(off, tgt, dev)
            directed, iters = True, 38
            run = lambda: g.pagerank_directed(0.85, iters, 0.0, copy_result=False)  # noqa: E731
        else:
            if name == "rmat22":
                g = G.GpuGraph.generate_rmat(dev, 22, EDGE_FACTOR, *RMAT_ABC, seed=2)
            else:
                g = G.GpuGraph.generate_erdos_renyi(dev, 1 << 22, 16 << 22, seed=3)
            directed, iters = False, 50
            run = lambda: g.pagerank_array(0.85, iters, 0.0, copy_result=False)  # noqa: E731
        V, E = g.num_nodes, g.num_edges
        run()
        dev.set_kernel_timing(True)
        dev.reset_stats()
        r = run()
        ks = dev.kernel_stats()
        dev.set_kernel_timing(False)
        launches = ks["pr_rows"][0]
        rows_ms = sum(ks[k][1] for k in ("pr_rows", "pr_chunks") if k in ks)
        per_it = rows_ms / r["iterations"]
        probe = float(np.median([g.pagerank_gather_probe(directed, 20) for _ in range(3)]))
        out[name] = {
            "vertices": V, "in_csr_entries": E, "iterations": r["iterations"], "pr_rows_launches": launches,
            "spmv_ms_per_iteration": round(per_it, 4),
            "gather_probe_ms_per_pass": round(probe, 4),
            "spmv_over_probe": round(per_it / probe, 3) if probe else None,
            "spmv_gbs_algorithmic": round(pr_bytes(V, E) / (per_it / 1e3) / 1e9, 1),
            "probe_gbs_of_4E": round(4 * E / (probe / 1e3) / 1e9, 1) if probe else None,
        }
        del g
    return out


def run_transpose_breakdown(scale: int) -> dict:
    """Where the directed plan build goes: from_csr of the R-MAT directed copy
    (3 % dangling), then pagerank_directed for one iteration, which builds the
    transpose (keys, 3 radix passes of histogram + scan + scatter, split) and
    the relabelled plan; per-kernel CUDA-event times, median of 4 builds after
    one warm-up build. The graph is generated on the device first (its own
    radix passes come before the transpose's)."""
    import grafeo_cuda as G

    seed = {24: 5, 22: 2}.get(scale, 1)
    dev = G.GpuDevice(0)
    g0 = G.GpuGraph.generate_rmat(dev, scale, EDGE_FACTOR, *RMAT_ABC, seed=seed)
    csr = g0.to_csr()
    del g0
    off, tgt, n_dangling = directed_dangling_copy(csr.offsets, csr.targets, DANGLING, seed)
    del csr
    builds = []
    for rep in range(5):
        g = G.GpuGraph.from_csr(off, tgt, dev)
        dev.synchronize()
        dev.set_kernel_timing(True)
        dev.reset_stats()
        g.pagerank_directed(DAMPING, 1, TOLERANCE, copy_result=False)
        ks = dev.kernel_stats()
        dev.set_kernel_timing(False)
        del g
        if rep:
            builds.append({k: v[1] for k, v in ks.items() if not k.startswith(("pr_rows", "pr_chunks", "pr_finish"))})
    names = sorted({k for b in builds for k in b}, key=lambda k: -statistics.median(b.get(k, 0.0) for b in builds))
    kernels = {k: round(statistics.median(b.get(k, 0.0) for b in builds), 3) for k in names}
    return {
        "transpose_breakdown": f"R-MAT scale {scale} seed {seed} directed copy ({DANGLING:.0%} dangling): device ms "
                               "per kernel of the directed PageRank plan build, median of 4",
        "device": dev.name, "vertices": len(off) - 1, "csr_entries": len(tgt), "dangling_vertices": n_dangling,
        "kernel_ms": kernels, "total_kernel_ms": round(sum(kernels.values()), 3),
    }


def main():
    args = parse_args()
    if args.transpose_breakdown:
        print(json.dumps(run_transpose_breakdown(args.scale)), flush=True)
        return
    if args.bfs_breakdown:
        print(json.dumps(run_bfs_breakdown()), flush=True)
        return
    if args.pr_ceiling:
        print(json.dumps(run_pr_ceiling()), flush=True)
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
