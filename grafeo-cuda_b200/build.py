"""Builds libgrafeo_cuda.so in place for sm_100a.

Compiles every source under csrc/ with nvcc (`-gencode arch=compute_100a,code=sm_100a
-O3 -lineinfo`) into _build/, links the shared library into grafeo_cuda/ next to
the Python module, and rewrites manifest.toml (source SHA-256s, nvcc version,
target and flags). This replaces the reference's build.rs / xtask PTX flow
(crates/grafeo-cuda-algos/build.rs, build_support/ptx_common.rs:291-308,
xtask/src/main.rs): there the committed sm_70 PTX had to match the sources;
here the sm_100a cubin is always built from the sources and the manifest
records exactly what it was built from (checked by `manifest.py check`).

Usage: python grafeo-cuda_b200/build.py [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "grafeo_cuda", "libgrafeo_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-fvisibility=hidden,-O3",
]
LINK_FLAGS = ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-lgomp"]

sys.path.insert(0, HERE)
import manifest  # noqa: E402


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources() -> list[str]:
    return sorted(
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp"))
    )


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "grafeo_cuda.h"))
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def compile_one(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + headers() + [os.path.abspath(__file__)]):
        lang = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [nvcc()] + NVCC_FLAGS + lang + ["-I", INCLUDE, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + LINK_FLAGS + objs + ["-o", LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    manifest.write(manifest.render(NVCC_FLAGS))
    if verbose:
        print(f"built {LIB}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    build(force=a.force, jobs=a.j, verbose=True)


if __name__ == "__main__":
    main()
