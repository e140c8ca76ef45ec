"""Shared pytest setup.

Markers: `gpu` for tests that need a CUDA device (they are the parity tests
proper and call through the C ABI); everything else runs on the CPU.
"""
from __future__ import annotations

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "grafeo-cuda_b200")
for p in (PKG, ROOT, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def pins() -> dict:
    with open(os.path.join(GOLDEN, "reference_pins.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_graphs() -> list[dict]:
    with open(os.path.join(GOLDEN, "catalog.json")) as f:
        return json.load(f)["graphs"]


@pytest.fixture(scope="session")
def pagerank_variants() -> list[dict]:
    with open(os.path.join(GOLDEN, "pagerank_variants.json")) as f:
        return json.load(f)["graphs"]


@pytest.fixture(scope="session")
def device():
    import grafeo_cuda

    if grafeo_cuda.device_count() == 0:
        pytest.fail("no CUDA device: GPU tests need a B200")
    return grafeo_cuda.GpuDevice(0)
