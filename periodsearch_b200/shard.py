"""Sharding trial periods across GPUs (one process per GPU).

Trial periods are independent units (README.md:12 of the reference: "the
period interval can be divided into smaller parts"), so a multi-GPU scan gives each rank disjoint blocks of consecutive periods and
needs no collective on the data path: the only exchange is the final
ordered gather of the 48-byte records to the writer.  Blocks are dealt
round-robin (block b goes to rank b % world), which balances uneven
iteration counts better than one contiguous slice per rank.
"""
from __future__ import annotations

import numpy as np


def period_blocks(n_total: int, world: int, rank: int, block: int) -> list[tuple[int, int]]:
    """1-based inclusive (n_from, n_to) blocks of this rank."""
    if world < 1 or not (0 <= rank < world) or block < 1:
        raise ValueError("bad shard arguments")
    out = []
    b = rank
    while b * block < n_total:
        a = b * block + 1
        out.append((a, min(a + block - 1, n_total)))
        b += world
    return out


def merge_records(parts, n_total: int, dtype) -> np.ndarray:
    """parts: iterable of (n_from, records) from all ranks -> records of
    periods 1..n_total in order; every period must appear exactly once."""
    out = np.zeros(n_total, dtype=dtype)
    seen = np.zeros(n_total, dtype=bool)
    for n_from, rec in parts:
        sl = slice(n_from - 1, n_from - 1 + len(rec))
        if seen[sl].any():
            raise ValueError("period assigned twice")
        out[sl] = rec
        seen[sl] = True
    if not seen.all():
        raise ValueError("periods missing from the gather")
    return out
