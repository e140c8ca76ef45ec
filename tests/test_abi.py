"""The C ABI boundary (CPU only): the library loads, exports every function
declared in include/*.h, and the Python binding declares each of them."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import grafeo_cuda
from grafeo_cuda import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions() -> list[str]:
    names = []
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"GCU_API\s+[\w\s\*]+?\b(gcu_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_boundary():
    names = declared_functions()
    for required in (
        "gcu_device_create",
        "gcu_graph_from_csr",
        "gcu_triangle_count",
        "gcu_triangle_count_oriented",
        "gcu_bfs",
        "gcu_pagerank",
        "gcu_k_truss",
        "gcu_validate_csr",
    ):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_python_binding_covers_the_header():
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_only_the_c_abi_is_exported():
    """Internal C++ symbols stay hidden (-fvisibility=hidden)."""
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    ours = {s for s in exported if s.startswith("gcu_")}
    assert ours == set(declared_functions())
    assert not any(s.startswith("_ZN3gcu") for s in exported)


def test_version_and_device_count_do_not_need_a_gpu():
    assert grafeo_cuda.version().startswith("0.3.0")
    assert grafeo_cuda.device_count() >= 0
