"""GPU parity for PageRank's chunked rows on CSRs built to reach every case.

The row kernels split the relabelled in-CSR three ways: rows of 1024 or more
entries go to 1024-entry segments, rows without entries to their own phase,
and every other row to the stream of 256-entry chunks (grafeo-cuda_b200/csrc/
pagerank.cu, pr_chunks_kernel). There the rows are packed back to back: a row
may cross one or several chunk boundaries, the chunked region may start a few
entries into the first chunk (when the long rows' entries do not end on an
8-entry boundary), and a chunk can hold up to 256 rows of one entry each. The
lists below are built so that every one of those cases occurs, and the ranks
must stay within L1 1e-6 of the FP64 oracle run for the same iteration count
(pagerank.rs semantics: pull over the lists, degree = list length), for the
plain, directed and personalised forms.
"""
from __future__ import annotations

import numpy as np
import pytest

import grafeo_cuda as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
ITERS = 30


def csr_from_lengths(lengths, V, seed):
    """Row i holds lengths[i] distinct sorted targets drawn from [0, V)."""
    rng = np.random.default_rng(seed)
    offsets = np.zeros(len(lengths) + 1, dtype=np.uint32)
    offsets[1:] = np.cumsum(lengths)
    targets = np.concatenate(
        [np.sort(rng.choice(V, size=int(n), replace=False)) for n in lengths if n > 0]
        or [np.zeros(0, dtype=np.int64)]).astype(np.uint32)
    return offsets, targets


def lengths_for(case, rng):
    if case == "mixed":
        # long rows of odd lengths (the chunked region starts unaligned), rows
        # crossing chunks, rows of exactly 255 / 256 / 257 entries, one-entry
        # rows, empty rows
        parts = [[1027, 2003, 1500], rng.integers(1, 1024, 1500), np.ones(700, int), np.full(60, 256),
                 np.full(40, 255), np.full(40, 257), np.zeros(500, int), rng.integers(1, 8, 900)]
    elif case == "short_only":  # no long rows: the chunks start at entry 0
        parts = [rng.integers(1, 40, 4000), np.zeros(100, int)]
    elif case == "ones":  # 256 rows per chunk: row deltas up to 255
        parts = [np.ones(3000, int)]
    elif case == "long_only":  # no chunked rows at all
        parts = [np.full(6, 1100), np.zeros(10, int)]
    else:  # rows of 300-1023 entries: every row crosses at least one boundary
        parts = [rng.integers(300, 1024, 400)]
    lengths = np.concatenate([np.asarray(p, dtype=np.int64) for p in parts])
    # A row holds distinct targets below the vertex count: pad with empty rows.
    lengths = np.concatenate([lengths, np.zeros(max(0, int(lengths.max()) - len(lengths)), dtype=np.int64)])
    rng.shuffle(lengths)
    return lengths


def symmetrised(offsets, targets):
    """The CSR with every entry mirrored, lists sorted and deduplicated."""
    V = len(offsets) - 1
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(offsets.astype(np.int64)))
    dst = targets.astype(np.int64)
    keys = np.unique(np.concatenate([src * V + dst, dst * V + src]))
    s_off = np.zeros(V + 1, dtype=np.uint32)
    s_off[1:] = np.cumsum(np.bincount(keys // V, minlength=V))
    return s_off, (keys % V).astype(np.uint32)


@pytest.mark.parametrize("case", ["mixed", "short_only", "ones", "long_only", "crossing"])
def test_chunked_rows_match_the_fp64_oracle(device, case):
    """The crafted lists are the in-lists of a directed graph (its out-CSR is
    their transpose), so directed PageRank pulls over exactly them; the plain
    form runs on the lists symmetrised (rank mass conserved in both)."""
    rng = np.random.default_rng(11)
    lengths = lengths_for(case, rng)
    V = len(lengths)
    in_off, in_tgt = csr_from_lengths(lengths, V, 5)
    out_off, out_tgt = O.transpose(in_off, in_tgt)
    gd = G.GpuGraph.from_csr(out_off, out_tgt, device)

    rd = gd.pagerank_directed(0.85, ITERS, 0.0)
    refd = O.pagerank_directed(out_off, out_tgt, 0.85, ITERS, 0.0)
    assert rd["iterations"] == ITERS
    assert np.abs(rd["ranks"].astype(np.float64) - refd["ranks"]).sum() <= L1_TOL, case

    seeds = rng.choice(V, size=5, replace=False)
    rp = gd.personalized_pagerank(seeds, 0.85, ITERS, 0.0, directed=True)
    refp = O.pagerank_directed(out_off, out_tgt, 0.85, ITERS, 0.0, tele=O.seed_vector(V, seeds))
    assert np.abs(rp["ranks"].astype(np.float64) - refp["ranks"]).sum() <= L1_TOL, case

    # Deterministic: the same ranks bit for bit on a second run.
    assert np.array_equal(gd.pagerank_directed(0.85, ITERS, 0.0)["ranks"], rd["ranks"])

    s_off, s_tgt = symmetrised(in_off, in_tgt)
    gs = G.GpuGraph.from_csr(s_off, s_tgt, device)
    r = gs.pagerank_array(0.85, ITERS, 0.0)
    ref = O.pagerank(s_off, s_tgt, 0.85, ITERS, 0.0)
    assert np.abs(r["ranks"].astype(np.float64) - ref["ranks"]).sum() <= L1_TOL, case
