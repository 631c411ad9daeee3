"""Sharding trial periods across GPUs (one process per GPU).

Trial periods are independent units (README.md:12 of the reference: "the
period interval can be divided into smaller parts"), so a multi-GPU scan gives each rank disjoint blocks of consecutive periods and
needs no collective on the data path: the only exchange is the final
ordered gather of the 48-byte records to the writer.  Blocks are dealt
round-robin (block b goes to rank b % world), which balances uneven
iteration counts better than one contiguous slice per rank.

The same partition is used by the executable (`period_search_b200 --shard
K/N`, then `--merge N`), by `scan_distributed` (one process per GPU under
torch.distributed) and by bench.py's per-rank batches.
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


def write_output(path: str, records: np.ndarray, conw_r: float, escl: float) -> None:
    """period_search_out of a whole scan, in the reference's format
    (period_search_BOINC.cpp:926-931): the first line carries conw_r escl^2
    in the dark-facet column."""
    from . import format_record

    with open(path, "w") as f:
        for i, r in enumerate(records):
            f.write(format_record(r, first_line=(i == 0), conw_line=conw_r * escl * escl))


def scan_distributed(source, block: int, out_path: str | None = None, group=None) -> np.ndarray:
    """Scan every trial period of one asteroid across the ranks of a
    torch.distributed process group (one process per GPU) and return the
    records of periods 1..n_periods in order on every rank.

    `source` is the rank's scan context after its convexity pre-pass: a
    periodsearch_b200.PeriodSearch on the rank's own GPU (every rank runs the
    same deterministic pre-pass, so no conw_r has to be sent), or any object
    with `n_periods`, `conw_r`, `escl` and `scan(n_from, n_to)`.  Each rank
    scans its round-robin blocks (period_blocks), the records are gathered
    once (48 bytes per period; no collective on the data path), merged and,
    on rank 0, written to `out_path` like an unsharded run."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = [(a, np.asarray(source.scan(a, b))) for a, b in period_blocks(source.n_periods, world, rank, block)]
    gathered = [None] * world
    dist.all_gather_object(gathered, (float(source.conw_r), mine), group=group)
    if any(c != gathered[0][0] for c, _ in gathered):
        raise ValueError("ranks disagree on conw_r")
    from . import RECORD_DTYPE

    merged = merge_records([p for _, parts in gathered for p in parts], source.n_periods, RECORD_DTYPE)
    if out_path and rank == 0:
        write_output(out_path, merged, source.conw_r, source.escl)
    return merged
