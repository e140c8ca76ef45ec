"""Kernel source manifest: what the sm_100a library is built from.

Replaces the reference's `kernels/ptx/manifest.toml` + `cargo xtask
check-ptx/regenerate-ptx` (xtask/src/main.rs:47-190,
build_support/ptx_common.rs:55-78). The reference committed sm_70 PTX and
checked that it matched the `.cu` files; here nothing compiled is committed,
so the manifest records, per source file, the SHA-256 of its text with CRLF
normalised to LF, plus the nvcc version, the target and the flags. `check`
fails when a source changed without the manifest being regenerated (which
`build.py` does on every build).

Usage: python grafeo-cuda_b200/manifest.py check|regenerate
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PATH = os.path.join(HERE, "manifest.toml")
TARGET = "sm_100a"


def source_files() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h")))


def sha256_lf(path: str) -> str:
    with open(path, "rb") as f:
        data = f.read().replace(b"\r\n", b"\n")
    return hashlib.sha256(data).hexdigest()


def nvcc_version() -> str:
    """Parses `release X.Y, VX.Y.Z` from `nvcc --version`."""
    try:
        out = subprocess.run(["nvcc", "--version"], capture_output=True, text=True).stdout
    except OSError:
        return "unknown"
    return parse_nvcc_version(out)


def parse_nvcc_version(text: str) -> str:
    m = re.search(r"V(\d+\.\d+\.\d+)", text)
    return m.group(1) if m else "unknown"


def render(flags: list[str]) -> str:
    lines = [
        "# Generated by grafeo-cuda_b200/build.py. Do not edit by hand.",
        "# Hashes are SHA-256 of the files with CRLF line endings normalized to LF.",
        f'nvcc = "{nvcc_version()}"',
        f'target = "{TARGET}"',
        "flags = [" + ", ".join(f'"{f}"' for f in flags) + "]",
        "",
    ]
    for name in source_files():
        lines.append(f"[sources.{name.replace('.', '_')}]")
        lines.append(f'file = "{name}"')
        lines.append(f'sha256 = "{sha256_lf(os.path.join(CSRC, name))}"')
        lines.append("")
    return "\n".join(lines)


def parse(text: str) -> dict:
    """Minimal TOML subset reader for this file's own format."""
    out: dict = {"sources": {}}
    section = None
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        if line.startswith("[") and line.endswith("]"):
            section = line[1:-1].split(".", 1)[1]
            out["sources"][section] = {}
            continue
        key, _, value = line.partition("=")
        key, value = key.strip(), value.strip()
        if value.startswith("["):
            parsed = re.findall(r'"([^"]*)"', value)
        else:
            parsed = value.strip('"')
        if section is None:
            out[key] = parsed
        else:
            out["sources"][section][key] = parsed
    return out


def write(text: str) -> None:
    with open(PATH, "w", newline="\n") as f:
        f.write(text)


def check() -> list[str]:
    """Returns the list of problems (empty when the manifest is current)."""
    if not os.path.exists(PATH):
        return ["manifest.toml is missing"]
    with open(PATH) as f:
        m = parse(f.read())
    problems = []
    if m.get("target") != TARGET:
        problems.append(f"target is {m.get('target')}, expected {TARGET}")
    flags = m.get("flags", [])
    if "arch=compute_100a,code=sm_100a" not in flags:
        problems.append("flags do not build for sm_100a")
    listed = {v["file"]: v["sha256"] for v in m["sources"].values()}
    for name in source_files():
        digest = sha256_lf(os.path.join(CSRC, name))
        if name not in listed:
            problems.append(f"{name} is not in the manifest")
        elif listed[name] != digest:
            problems.append(f"{name} changed since the manifest was generated")
    for name in listed:
        if name not in source_files():
            problems.append(f"{name} is in the manifest but not in csrc/")
    return problems


def main() -> int:
    cmd = sys.argv[1] if len(sys.argv) > 1 else "check"
    if cmd == "regenerate":
        sys.path.insert(0, HERE)
        from build import NVCC_FLAGS

        write(render(NVCC_FLAGS))
        print(f"wrote {PATH}")
        return 0
    problems = check()
    for p in problems:
        print(p)
    return 1 if problems else 0


if __name__ == "__main__":
    sys.exit(main())
