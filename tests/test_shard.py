"""Multi-process period sharding on CPU: two gloo ranks scan disjoint period
blocks (with the CPU oracle standing in for the per-rank GPU scan) and the
ordered gather on rank 0 reproduces the single-process scan exactly."""
import os
import socket

import numpy as np
import pytest

from conftest import REPO, golden_path


def test_period_blocks_cover_once():
    from periodsearch_b200.shard import period_blocks

    for n_total in (1, 7, 200, 39153):
        for world in (1, 2, 3, 8):
            for block in (1, 5, 592):
                seen = np.zeros(n_total, int)
                for r in range(world):
                    for a, b in period_blocks(n_total, world, r, block):
                        seen[a - 1:b] += 1
                assert np.all(seen == 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, path, conw_r, out_path):
    import sys

    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import torch.distributed as dist

    import pso
    from periodsearch_b200.shard import merge_records, period_blocks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    o = pso.Oracle(path)
    o.set_conw_r(conw_r)
    mine = [(a, o.scan(a, b)) for a, b in period_blocks(o.n_periods, world, rank, 1)]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        parts = [p for rp in gathered for p in rp]
        np.save(out_path, merge_records(parts, o.n_periods, pso.RECORD_DTYPE))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_scan_matches_single_process(oracle_lib, tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    path = golden_path("tiny")
    o = oracle_lib.Oracle(path)
    conw_r = o.conw_r
    o.set_conw_r(conw_r)
    single = o.scan(1, o.n_periods)
    out = str(tmp_path / "merged.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), path, conw_r, out), nprocs=2, join=True,
                       start_method="spawn")
    merged = np.load(out)
    for k in single.dtype.names:
        assert np.array_equal(merged[k], single[k]), k
