"""The radix sort's scatter arithmetic, restated on the host.

csrc/sort.cu sorts 64-bit keys by 8-bit digits, least significant first. One
pass is three steps:

1. `radix_hist_kernel` counts the digits of every CTA range of
   kTilesPerCta x kSortTile keys (digit-major).
2. One exclusive scan turns those counts into each (digit, CTA) output base.
3. `radix_scatter_smem_kernel` walks its CTA's tiles in order. Each warp ranks
   the keys of its slice round by round, 32 lanes at a time. Equal-digit lane
   masks come from 8 ballots, and the rank, the lane count and the first-lane
   flag are packed into 16 bits per key. One block scan gives each warp's
   offset inside each digit and each digit's start inside the tile. The keys
   are placed in digit order and written to `base[digit] + (j - start[digit])`.
   The digit bases advance by the tile's counts.

These tests repeat that arithmetic step for step: the ballots, the packed
words, the counters and the carried bases. They check that one pass equals a
stable sort by its digit and that the 3-pass sort equals numpy's stable
argsort. The inputs are ragged: the last CTA range and the last tile are
partial, and lanes past the end have no key. They include a run where all 32
lanes of a round share one digit, so the count field's 6 bits are exercised.
"""
from __future__ import annotations

import numpy as np
import pytest

RADIX = 256
FULL = 0xFFFFFFFF
LANES = np.arange(32, dtype=np.uint64)


def ballot(pred: np.ndarray) -> int:
    return int((pred.astype(np.uint64) << LANES).sum())


def popc(x: int) -> int:
    return bin(x & FULL).count("1")


def same_digit_lanes(d: np.ndarray) -> list[int]:
    """Per lane, the mask of lanes holding the same digit (RADIX: no key), as
    sort.cu's same_digit_lanes builds it from one ballot per digit bit."""
    none = ballot(d == RADIX)
    masks = [none ^ (0 if d[l] == RADIX else FULL) for l in range(32)]
    for b in range(8):
        pred = (d >> b) & 1
        bits = ballot(pred == 1)
        masks = [m & (bits if pred[l] else ~bits & FULL) for l, m in enumerate(masks)]
    return masks


def scatter_pass(keys: np.ndarray, shift: int, tile_keys: int, tiles_per_cta: int, warps: int = 8) -> np.ndarray:
    n = len(keys)
    cta_keys = tile_keys * tiles_per_cta
    nctas = -(-n // cta_keys)
    digit = ((keys >> np.uint64(shift)) & np.uint64(0xFF)).astype(np.int64)
    # radix_hist_kernel: digit counts per CTA range, digit-major.
    hist = np.zeros((RADIX, nctas), dtype=np.int64)
    for b in range(nctas):
        hist[:, b] = np.bincount(digit[b * cta_keys:(b + 1) * cta_keys], minlength=RADIX)
    bases = np.concatenate([[0], np.cumsum(hist.ravel())[:-1]]).reshape(RADIX, nctas)
    slice_keys = tile_keys // warps
    per_lane = slice_keys // 32
    out = np.full(n, np.iinfo(np.uint64).max, dtype=np.uint64)
    written = np.zeros(n, dtype=bool)
    below = [(1 << l) - 1 for l in range(32)]
    for b in range(nctas):
        s_base = bases[:, b].copy()
        for t in range(tiles_per_cta):
            tile0 = b * cta_keys + t * tile_keys
            if tile0 >= n:
                break
            s_woff = np.zeros((warps, RADIX), dtype=np.int64)
            info = {}
            lane_digits = {}
            # Counting pass: first lanes add their digit's count; every lane
            # keeps rank | count << 5 | first << 11.
            for w in range(warps):
                for q in range(per_lane):
                    idx = tile0 + w * slice_keys + q * 32 + np.arange(32)
                    d = np.where(idx < n, digit[np.minimum(idx, n - 1)], RADIX)
                    lane_digits[w, q] = d
                    masks = same_digit_lanes(d)
                    words = []
                    for l in range(32):
                        m = masks[l]
                        first = d[l] < RADIX and l == (m & -m).bit_length() - 1
                        if first:
                            s_woff[w, d[l]] += popc(m)
                        words.append(popc(m & below[l]) | (popc(m) << 5) | ((1 << 11) if first else 0))
                    # Two keys' words per 32-bit register: even rounds low, odd rounds high.
                    if q % 2 == 0:
                        info[w, q // 2] = list(words)
                    else:
                        info[w, q // 2] = [lo | (hi << 16) for lo, hi in zip(info[w, q // 2], words)]
            # Block scan: warps' exclusive offsets inside each digit, digits'
            # exclusive starts inside the tile, the tile's digit totals.
            tot = s_woff.sum(axis=0)
            s_woff = np.cumsum(s_woff, axis=0) - s_woff
            s_start = np.cumsum(tot) - tot
            s_keys = np.full(tile_keys, np.iinfo(np.uint64).max, dtype=np.uint64)
            # Placing pass: from the packed words only.
            for w in range(warps):
                for q in range(per_lane):
                    d = lane_digits[w, q]
                    words = [(x >> (16 if q % 2 else 0)) & 0xFFFF for x in info[w, q // 2]]
                    for l in range(32):
                        if d[l] < RADIX:
                            v = words[l]
                            s_keys[s_start[d[l]] + s_woff[w, d[l]] + (v & 31)] = keys[tile0 + w * slice_keys + q * 32 + l]
                    for l in range(32):
                        v = words[l]
                        if (v >> 11) & 1:
                            s_woff[w, d[l]] += (v >> 5) & 63
            valid = min(tile_keys, n - tile0)
            for j in range(valid):
                k = s_keys[j]
                dd = int((k >> np.uint64(shift)) & np.uint64(0xFF))
                pos = s_base[dd] + (j - s_start[dd])
                assert not written[pos], "two keys written to one position"
                out[pos] = k
                written[pos] = True
            s_base += tot
    assert written.all(), "a position left unwritten"
    return out


def radix_sort(keys: np.ndarray, low_bit: int, high_bit: int, tile_keys: int, tiles_per_cta: int) -> np.ndarray:
    for shift in range(low_bit, high_bit, 8):
        keys = scatter_pass(keys, shift, tile_keys, tiles_per_cta)
    return keys


def stable_by_digit(keys: np.ndarray, shift: int) -> np.ndarray:
    digit = (keys >> np.uint64(shift)) & np.uint64(0xFF)
    return keys[np.argsort(digit, kind="stable")]


@pytest.mark.parametrize("n", [1, 31, 2048, 4465, 70001])
def test_one_pass_is_a_stable_sort_by_its_digit(n):
    # Shipped shape: 256 threads x 8 keys per lane (2,048-key tiles), 16 tiles per CTA.
    rng = np.random.default_rng(n)
    keys = (rng.integers(0, 1 << 24, n, dtype=np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    for shift in (32, 40):
        assert np.array_equal(scatter_pass(keys, shift, 2048, 16), stable_by_digit(keys, shift))


def test_full_width_digit_runs():
    # Every lane of a round holds digit 0, then a short tail of another digit.
    n = 5000
    digits = np.zeros(n, dtype=np.uint64)
    digits[-37:] = 200
    keys = (digits << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    assert np.array_equal(scatter_pass(keys, 32, 2048, 16), stable_by_digit(keys, 32))


@pytest.mark.parametrize("tile_keys,tiles_per_cta", [(2048, 16), (2048, 2), (4096, 1)])
def test_transpose_keys_sort_keeps_sources_ascending(tile_keys, tiles_per_cta):
    # (target << 32 | source) keys of a skewed random CSR, in source order,
    # sorted by the 24 target bits as the transpose does.
    rng = np.random.default_rng(7)
    n = 9000
    targets = np.minimum(rng.zipf(1.6, n) - 1, (1 << 24) - 1).astype(np.uint64)
    sources = np.sort(rng.integers(0, 1 << 20, n)).astype(np.uint64)
    keys = (targets << np.uint64(32)) | sources
    got = radix_sort(keys, 32, 56, tile_keys, tiles_per_cta)
    want = keys[np.argsort(targets, kind="stable")]
    assert np.array_equal(got, want)
    hi = got >> np.uint64(32)
    lo = got & np.uint64(FULL)
    same = hi[1:] == hi[:-1]
    assert np.all(lo[1:][same] >= lo[:-1][same]), "an in-list out of source order"
