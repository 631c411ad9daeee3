"""Batched scans (ps_batch_*): several asteroids with different point
counts, calibrated/relative mixes and per-fit LM convergence in one
persistent launch replayed from a CUDA graph.  Every fit runs exactly the
code of a single-asteroid scan, so the records must be bit-identical to
scanning each asteroid on its own; through the batch the scans still match
the reference."""
import numpy as np
import pytest

from conftest import golden_path
from test_gpu_parity import _read_full, check_records, perturbation_spread

pytestmark = pytest.mark.gpu


def _asteroids(tmp_path, n=4):
    from periodsearch_b200 import synth

    paths = []
    for i in range(n):
        w = synth.make_workload(f"b{i}", 100 + i, dense_lcs=1 + i, dense_pts=15 + 10 * i, sparse_pts=20 * (i % 3),
                                years=4, true_lmax=3, fit_lmax=3, nrows=4, noise=0.02, n_periods=3 + i,
                                stop_condition=0.001, n_iter_min=5)
        paths.append(synth.write_input(w, str(tmp_path / f"a{i}")))
    return paths


@pytest.mark.parametrize("form", ["fp64", "fast", "mixed"])
def test_batch_equals_single_scans(native, tmp_path, form):
    ps = native
    fid = {"fp64": ps.PS_FORM_FP64, "fast": ps.PS_FORM_FAST, "mixed": ps.PS_FORM_MIXED}[form]
    ctxs = [ps.PeriodSearch(p, form=fid) for p in _asteroids(tmp_path)]
    for c in ctxs:
        c.set_conw_r(c.conw_r * 4)
    batch = ps.PeriodSearchBatch(ctxs)
    for rng in ([(1, c.n_periods) for c in ctxs], [(2, 2), (1, 3), (3, 4), (1, 1)]):
        n_from = [a for a, _ in rng]
        n_to = [min(b, c.n_periods) for (_, b), c in zip(rng, ctxs)]
        got = batch.scan(n_from, n_to)
        for c, a, b, g in zip(ctxs, n_from, n_to, got):
            want = c.scan(a, b)
            for k in want.dtype.names:
                assert np.array_equal(g[k], want[k]), (form, k)
    busy, done = batch.fit_times()
    assert np.all(busy > 0) and np.all(done > 0)
    assert np.all(done <= busy.sum() + 1e-3)  # no asteroid finishes after all fits ran back to back
    batch.close()
    for c in ctxs:
        c.close()


def test_batch_matches_reference(native):
    ps = native
    names = ["c1", "c1_conv"]
    ctxs = []
    for name in names:
        c = ps.PeriodSearch(golden_path(name), form=ps.PS_FORM_FAST)
        c.precalc()
        ctxs.append(c)
    refs = [_read_full(golden_path(n, "ref_out.full")) for n in names]
    batch = ps.PeriodSearchBatch(ctxs)
    got = batch.scan([1, 1], [len(r) for r in refs])
    for name, g, r in zip(names, got, refs):
        check_records(g, r, perturbation_spread(name, r), name)
    batch.close()
    for c in ctxs:
        c.close()
