"""Host-side logic of the library (CPU only): CSR validation messages, CSR
builders, the TSV parser, the synthetic generators and the source manifest.

Mirrors crates/grafeo-cuda-core/tests/csr_export.rs (validation, builders,
TSV parser) and xtask/src/main.rs tests (manifest).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import grafeo_cuda as G
from grafeo_cuda import GrafeoCudaError
from oracle import oracle as O

import graphs


def test_validate_accepts_well_formed_csr(pins):
    for case in pins["validate_accepts"]:
        G.validate_csr(case["offsets"], case["targets"])


def test_validate_rejects_malformed_csr_with_reference_messages(pins):
    for case in pins["validate_messages"]:
        with pytest.raises(GrafeoCudaError) as e:
            G.validate_csr(case["offsets"], case["targets"])
        assert e.value.status == G.ERR_INVALID_CSR
        assert case["contains"] in str(e.value), (case, str(e.value))
        assert str(e.value).startswith("invalid CSR: ")


def test_validate_exact_messages():
    cases = {
        ((1, 1), (0,)): "invalid CSR: offsets[0] must be 0, got 1",
        ((0, 2), (1,)): "invalid CSR: offsets[1] is 2 but targets has 1 entries",
        ((0, 2, 1, 2), (1, 2)): "invalid CSR: offsets decrease at node 1: 2 then 1",
        ((0, 1, 1), (2,)): "invalid CSR: node 0 has neighbor 2, but there are only 2 nodes",
        ((0, 2, 2), (1, 1)): "invalid CSR: neighbor list of node 0 is not strictly increasing"
        + " " * 22 + "(1 then 1)",
        ((), ()): "invalid CSR: offsets must have num_nodes + 1 entries, got an empty array",
    }
    for (o, t), msg in cases.items():
        with pytest.raises(GrafeoCudaError) as e:
            G.validate_csr(list(o), list(t))
        assert str(e.value) == msg


def test_csr_arrays_validate_checks_declared_counts():
    """csr_export.rs(tests):553-562."""
    csr = G.from_edge_pairs([(0, 1)], 2, True)
    csr.validate()
    csr.num_nodes = 3
    with pytest.raises(GrafeoCudaError):
        csr.validate()
    csr.num_nodes = 2
    csr.num_edges = 1
    with pytest.raises(GrafeoCudaError):
        csr.validate()


def test_builders_match_reference_examples(pins):
    for b in pins["builders"]:
        if b["call"] == "from_edge_pairs":
            c = G.from_edge_pairs(b["edges"], b["num_nodes"], b["symmetric"])
        else:
            c = G.from_edge_pairs_oriented(b["edges"], b["num_nodes"])
        assert c.offsets.tolist() == b["offsets"] and c.targets.tolist() == b["targets"], b


@pytest.mark.parametrize("seed", range(24))
def test_builders_match_oracle_on_random_pairs(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(1, 20))
    raw = rng.integers(0, n, size=(int(rng.integers(0, 80)), 2))
    for sym in (False, True):
        c = G.from_edge_pairs(raw, n, sym)
        o, t = O.from_edge_pairs(raw, n, sym)
        assert c.offsets.tolist() == o.tolist() and c.targets.tolist() == t.tolist()
        c.validate()
    c = G.from_edge_pairs_oriented(raw, n)
    o, t = O.from_edge_pairs_oriented(raw, n)
    assert c.offsets.tolist() == o.tolist() and c.targets.tolist() == t.tolist()
    c.validate()


def test_builders_reject_out_of_range_nodes():
    with pytest.raises(GrafeoCudaError) as e:
        G.from_edge_pairs([(5, 0)], 3, True)
    assert e.value.status == G.ERR_EXPORT
    with pytest.raises(GrafeoCudaError):
        G.from_edge_pairs_oriented([(0, 9)], 3)


def test_tsv_parser(tmp_path, pins):
    for i, case in enumerate(pins["tsv"]):
        p = tmp_path / f"g{i}.tsv"
        p.write_text(case["text"])
        edges, n = G.parse_tsv_to_edges(p)
        assert [list(e) for e in edges] == case["edges"] and n == case["num_nodes"], case


def test_tsv_parser_reports_missing_file(tmp_path):
    with pytest.raises(GrafeoCudaError) as e:
        G.parse_tsv_to_edges(tmp_path / "definitely-missing.tsv")
    assert e.value.status == G.ERR_EXPORT


def test_rmat_generator_is_deterministic_and_clean():
    a = G.generate_rmat(10, 8, seed=7)
    b = G.generate_rmat(10, 8, seed=7)
    c = G.generate_rmat(10, 8, seed=8)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.targets, b.targets)
    assert not np.array_equal(a.targets, c.targets)
    a.validate()
    assert a.num_nodes == 1024
    # symmetric, loop-free
    src = np.repeat(np.arange(a.num_nodes), np.diff(a.offsets))
    assert not np.any(src == a.targets)
    fwd = set(zip(src.tolist(), a.targets.tolist()))
    assert all((v, u) in fwd for u, v in fwd)
    # R-MAT skew: vertex 0 (all-zero bits, quadrant a) is the largest hub
    deg = np.diff(a.offsets)
    assert deg[0] == deg.max()


def test_rmat_scale14_config_shape():
    """The small config: 16,384 vertices, about 426k CSR entries, hub at 0."""
    g = G.generate_rmat(14, 16, 0.57, 0.19, 0.19, seed=1)
    assert g.num_nodes == 16384
    assert 400_000 < g.num_edges < 450_000
    assert g.num_edges % 2 == 0


def test_erdos_renyi_generator():
    g = G.generate_erdos_renyi(4096, 16 * 4096, seed=3)
    g.validate()
    deg = np.diff(g.offsets)
    assert 30 < deg.mean() < 33  # average degree ~32 after dropping repeats
    src = np.repeat(np.arange(g.num_nodes), deg)
    assert not np.any(src == g.targets)


def test_python_list_conversion_rejects_out_of_range():
    with pytest.raises(OverflowError):
        G.validate_csr([0, -1], [])
    with pytest.raises(OverflowError):
        G.validate_csr([0, 2**32], [])


def test_no_device_is_reported_like_the_reference():
    if G.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(GrafeoCudaError) as e:
        G.GpuDevice(0)
    assert e.value.status == G.ERR_NO_DEVICE
    assert str(e.value) == "no CUDA device found"


def test_manifest_is_current():
    import manifest

    assert manifest.check() == []


def test_manifest_parses_nvcc_version():
    import manifest

    text = "nvcc: NVIDIA (R) Cuda compiler driver\nCuda compilation tools, release 12.9, V12.9.86\n"
    assert manifest.parse_nvcc_version(text) == "12.9.86"
    assert manifest.parse_nvcc_version("garbage") == "unknown"


def test_manifest_roundtrip():
    import manifest

    text = manifest.render(["-gencode", "arch=compute_100a,code=sm_100a"])
    parsed = manifest.parse(text)
    assert parsed["target"] == "sm_100a"
    files = {v["file"] for v in parsed["sources"].values()}
    assert "pagerank.cu" in files and "bfs.cu" in files


def test_wide_frontier_fixture_shape():
    n, pairs, expected = graphs.wide_frontier(width=10, depth=4)
    assert n == 42 and len(expected) == n
    c = G.from_edge_pairs(pairs, n, True)
    r = O.bfs(c.offsets, c.targets, 0)
    assert r["distances"].tolist() == expected.tolist() and r["max_depth"] == 5


def test_schedule_margin_matches_the_device_constant():
    """The Python evaluation of the learned schedule applies the same margin
    over the fixed rule as the device's decide kernels."""
    import os
    import re

    from grafeo_cuda import schedule

    src = open(os.path.join(os.path.dirname(__file__), "..", "grafeo-cuda_b200", "csrc", "sched.cuh")).read()
    value = float(re.search(r"kSchedMarginLog2\s*=\s*([0-9.]+)f", src).group(1))
    assert value == schedule.MARGIN_LOG2
