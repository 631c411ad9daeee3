"""Multi-process period sharding on CPU: two gloo ranks run the product's
distributed scan (periodsearch_b200.shard.scan_distributed: round-robin
blocks, one gather, merge, output writer) with the CPU oracle standing in for
each rank's GPU scan context, and reproduce the single-process scan and its
period_search_out exactly."""
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


def _rank_main(rank, world, port, path, conw_r, out_path, text_path):
    import sys

    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import torch.distributed as dist

    import pso
    from periodsearch_b200.shard import scan_distributed

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    o = pso.Oracle(path)
    o.set_conw_r(conw_r)
    merged = scan_distributed(o, block=3, out_path=text_path)
    if rank == 0:
        np.save(out_path, merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_scan_matches_single_process(oracle_lib, native, tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    from periodsearch_b200.shard import write_output

    path = golden_path("tiny")
    o = oracle_lib.Oracle(path)
    conw_r = o.conw_r
    o.set_conw_r(conw_r)
    single = o.scan(1, o.n_periods)
    out = str(tmp_path / "merged.npy")
    text = str(tmp_path / "period_search_out")
    mp.start_processes(_rank_main, args=(2, _free_port(), path, conw_r, out, text), nprocs=2, join=True,
                       start_method="spawn")
    merged = np.load(out)
    for k in single.dtype.names:
        assert np.array_equal(merged[k], single[k]), k
    want = str(tmp_path / "single_out")
    write_output(want, single, conw_r, o.escl)
    assert open(text).read() == open(want).read()
    assert len(open(text).read().splitlines()) == o.n_periods


def test_merge_rejects_overlap_and_gaps():
    from periodsearch_b200 import RECORD_DTYPE
    from periodsearch_b200.shard import merge_records

    r = np.zeros(2, dtype=RECORD_DTYPE)
    with pytest.raises(ValueError):
        merge_records([(1, r), (2, r)], 3, RECORD_DTYPE)
    with pytest.raises(ValueError):
        merge_records([(1, r)], 3, RECORD_DTYPE)
