"""PageRank's chunked rows, restated on the host.

csrc/pagerank.cu reads the rows of 1 to 1023 entries of its relabelled
in-CSR as a stream of 256-entry chunks. The chunks start at `origin`, the
first chunked entry rounded down to 8. It works in three places:

* The plan: `pr_chunk_rows_kernel` gives every chunk its first row and flags
  the rows split between chunks. `pr_split_rows_kernel` lists those rows as
  (row, first chunk, last chunk). `pr_perm_fill_kernel` stores each entry's
  row as a byte, its row minus the chunk's first row.
* `pr_chunks_kernel`: one warp per chunk, 8 consecutive entries per lane.
  Each lane sums its runs of equal rows. A run that is neither the lane's
  first nor its last is a whole row, finished there. The lanes' last runs are
  joined by a segmented inclusive scan. A lane finishes a row where the row's
  run ends, except for the parts of rows that cross chunks. Those go to
  chunk_part[2c] (chunk c's first row, begun in an earlier chunk) and to
  chunk_part[2c + 1] (its last row, going on into the next chunk, or the
  whole chunk when one row covers it).
* `pr_finish_kernel`: a split row's sum is its first chunk's [2c + 1], the
  [2c + 1] of every chunk it covers whole, and its last chunk's [2c].

These tests repeat the arithmetic lane by lane, shuffles and scan steps
included. The contributions are small integers, so every sum is exact. They
check that every chunked row is finished exactly once, with the sum of its
entries, and that the finishing kernel reads only the part slots the chunk
kernel wrote. The row-length mixes are: random, all ones, all 1023, rows of
exactly 256, chunk-aligned and unaligned starts, and an end on a chunk
boundary.
"""
from __future__ import annotations

import numpy as np
import pytest

CHUNK = 256
NO_ROW = 0xFFFFFFFF


def chunk_plan(poff: np.ndarray, r0: int, r1: int):
    """The plan's chunk arrays for chunked rows [r0, r1) (pr_chunk_rows_kernel,
    pr_split_rows_kernel and the delta bytes of pr_perm_fill_kernel)."""
    lo, hi = int(poff[r0]), int(poff[r1])
    origin = lo & ~7
    n_chunks = -(-(hi - origin) // CHUNK)
    chunk_row = np.full(n_chunks, -1, dtype=np.int64)
    split = []
    for r in range(r0, r1):
        s, e = int(poff[r]) - origin, int(poff[r + 1]) - origin
        assert e > s, "every chunked row has entries"
        c_first, c_last = s // CHUNK, (e - 1) // CHUNK
        for c in range(0 if r == r0 else -(-s // CHUNK), c_last + 1):
            chunk_row[c] = r
        if c_first != c_last:
            split.append((r, c_first, c_last))
    assert (chunk_row >= 0).all(), "a chunk without a first row"
    delta = np.zeros(n_chunks * CHUNK, dtype=np.int64)
    for r in range(r0, r1):
        for k in range(int(poff[r]), int(poff[r + 1])):
            rel = k - origin
            delta[rel] = r - chunk_row[rel // CHUNK]
    assert delta.max() < 256, "a row delta past one byte"
    return lo, hi, origin, n_chunks, chunk_row, delta, split


def shfl_up(x: list, d: int) -> list:
    return [x[l - d] if l >= d else x[l] for l in range(32)]


def shfl_down(x: list, d: int) -> list:
    return [x[l + d] if l + d < 32 else x[l] for l in range(32)]


def run_chunks(poff, vals, r0, r1):
    """pr_chunks_kernel then the split-row part of pr_finish_kernel; returns
    {row: sum} with every finish recorded once."""
    lo, hi, origin, n_chunks, chunk_row, delta, split = chunk_plan(poff, r0, r1)
    finished: dict[int, float] = {}
    part: dict[int, float] = {}

    def finish(r, s):
        assert r not in finished, f"row {r} finished twice"
        finished[r] = s

    def put(slot, s):
        assert slot not in part, f"part slot {slot} written twice"
        part[slot] = s

    for c in range(n_chunks):
        e0 = origin + c * CHUNK
        rbase = int(chunk_row[c])
        first_split = int(poff[rbase]) < e0
        rows, accs, heads, multis = [], [], [], []
        for lane in range(32):
            eb = e0 + 8 * lane
            row = [rbase + int(delta[eb + i - origin]) if lo <= eb + i < hi else NO_ROW for i in range(8)]
            val = [float(vals[eb + i]) if lo <= eb + i < hi else 0.0 for i in range(8)]
            head, acc, multi = 0.0, 0.0, False
            for i in range(8):
                acc += val[i]
                if i < 7 and row[i + 1] != row[i]:
                    if not multi:
                        head, multi = acc, True
                    else:
                        assert row[i] != NO_ROW, "a middle run without a row"
                        finish(row[i], acc)
                    acc = 0.0
            rows.append(row)
            accs.append(acc)
            heads.append(head)
            multis.append(multi)
        rlast = rows[31][7]
        last_split = rlast != NO_ROW and int(poff[rlast + 1]) > e0 + CHUNK
        rf = [rows[l][0] for l in range(32)]
        rl = [rows[l][7] for l in range(32)]
        prev_last = shfl_up(rl, 1)
        next_first = shfl_down(rf, 1)
        carry_in = [l > 0 and prev_last[l] == rf[l] for l in range(32)]
        flag = [multis[l] or not carry_in[l] for l in range(32)]
        S = list(accs)
        d = 1
        while d < 32:
            su, fu = shfl_up(S, d), shfl_up(flag, d)
            S = [S[l] + su[l] if l >= d and not flag[l] else S[l] for l in range(32)]
            flag = [flag[l] or fu[l] if l >= d else flag[l] for l in range(32)]
            d <<= 1
        carry = shfl_up(S, 1)
        for lane in range(32):
            if multis[lane] and rf[lane] != NO_ROW:
                total = heads[lane] + (carry[lane] if carry_in[lane] else 0.0)
                if rf[lane] == rbase and first_split:
                    put(2 * c, total)
                else:
                    finish(rf[lane], total)
            continues = lane < 31 and next_first[lane] == rl[lane]
            if not continues and rl[lane] != NO_ROW:
                if lane == 31 and last_split:
                    put(2 * c + 1, S[lane])
                elif rl[lane] == rbase and first_split:
                    put(2 * c, S[lane])
                else:
                    finish(rl[lane], S[lane])
    read = set()
    for r, c_first, c_last in split:
        slots = [2 * c_first + 1] + [2 * c + 1 for c in range(c_first + 1, c_last)] + [2 * c_last]
        for s in slots:
            assert s in part, f"part slot {s} read but never written"
            read.add(s)
        finish(r, sum(part[s] for s in slots))
    assert read == set(part), "a part slot written but never read"
    return finished


def layout(lengths, lo: int, seed: int):
    """poff for rows [r0, r1) of the given lengths starting at entry lo (the
    rows before r0 stand for the long rows), and integer contributions."""
    r0 = 3
    poff = np.zeros(r0 + len(lengths) + 1, dtype=np.int64)
    poff[: r0 + 1] = np.linspace(0, lo, r0 + 1).astype(np.int64)
    poff[r0 + 1:] = lo + np.cumsum(lengths)
    rng = np.random.default_rng(seed)
    vals = rng.integers(1, 64, int(poff[-1]) + CHUNK).astype(np.float64)
    return poff, vals, r0, r0 + len(lengths)


def check(lengths, lo, seed=0):
    poff, vals, r0, r1 = layout(np.asarray(lengths, dtype=np.int64), lo, seed)
    got = run_chunks(poff, vals, r0, r1)
    assert sorted(got) == list(range(r0, r1)), "a chunked row not finished"
    for r in range(r0, r1):
        assert got[r] == vals[poff[r]:poff[r + 1]].sum(), f"row {r}"


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("lo", [0, 1237, 4096])
def test_random_row_lengths(seed, lo):
    rng = np.random.default_rng(100 + seed)
    # Heavy-tailed lengths in 1..1023, like the degree classes below the long rows.
    lengths = np.minimum(1023, np.maximum(1, (rng.pareto(1.2, 400) * 4).astype(np.int64) + 1))
    check(lengths, lo, seed)


@pytest.mark.parametrize("lengths", [
    [1] * 3000,              # many rows per lane
    [1023] * 20,             # every row crosses several chunks
    [256] * 30,              # rows exactly one chunk long
    [7, 249, 256, 1, 511, 1023, 3, 300, 2, 2],
    [255, 1, 256, 512, 1],   # an end on a chunk boundary from an aligned start
])
@pytest.mark.parametrize("lo", [0, 5, 8, 256 + 3])
def test_row_length_mixes(lengths, lo):
    check(lengths, lo)
