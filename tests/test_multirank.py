"""The N > 1 path of bench.py on CPU: two gloo ranks on 127.0.0.1.

The graph paths run one replica per GPU with no data-path collective; the only
cross-rank steps are the barrier and the max/sum of the timings. These tests
check that plumbing and the reference arm's rank handling (rank 0 alone works
and prints; the other ranks exit 0 without work).
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["BENCH_ROOT"])
import bench
d = bench.Dist()
rank = d.rank
d.barrier()
mx = d.max(10.0 + rank)
sm = d.sum(1.0 + rank)
# One file per rank: two ranks printing to one pipe can interleave their lines.
with open(os.path.join(os.environ["OUT_DIR"], f"rank{rank}.json"), "w") as fh:
    json.dump({"rank": rank, "world": d.world, "max": mx, "sum": sm}, fh)
d.close()
"""


def run_torchrun(args, env_extra=None, timeout=300):
    env = dict(os.environ)
    env["BENCH_ROOT"] = ROOT
    env["CUDA_VISIBLE_DEVICES"] = ""
    if env_extra:
        env.update(env_extra)
    # A port picked free can be taken again before the rendezvous binds it:
    # retry on a fresh port when the launcher itself fails.
    for attempt in range(3):
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
               "--master-addr=127.0.0.1", f"--master-port={free_port()}"] + args
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout, cwd=ROOT)
        if r.returncode == 0 or not any(s in r.stderr for s in ("EADDRINUSE", "address already in use",
                                                                 "RendezvousConnectionError", "DistNetworkError")):
            return r
    return r


def test_dist_max_and_sum_over_two_gloo_ranks(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    r = run_torchrun([str(script)], env_extra={"OUT_DIR": str(tmp_path)})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in (0, 1)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    for x in lines:
        assert x["world"] == 2 and x["max"] == 11.0 and x["sum"] == 3.0


def test_reference_arm_prints_once_under_two_ranks():
    r = run_torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--scale", "10", "--steps", "1",
                      "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["unit"] == "GB/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
