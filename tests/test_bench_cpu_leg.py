"""bench.py's CPU legs (no GPU): a workload beyond the reference
application's static arrays (constants.h: MAX_N_FAC = 1000 facets,
MAX_N_OBS = 20000 points) is not handed to the compiled reference -- which
exits with status 2 on it -- but timed on the restatement, per model
evaluation; the c2 workload stays within the limits."""
import os
import sys

import pytest

from conftest import REPO

sys.path.insert(0, REPO)


def test_large_workload_uses_the_restatement(tmp_path):
    import bench

    p = bench.make_input(str(tmp_path), "c5")
    r, why = bench.ref_cpu_sample_or_none(p, 1)
    assert r is None
    assert "2048 facets" in why and "MAX_N_FAC" in why


def test_production_workload_fits_the_reference(tmp_path):
    import bench
    import pso

    p = bench.make_input(str(tmp_path), "c2")
    o = pso.Oracle(p)
    o.set_conw_r(o.conw_r)
    assert o.numfac <= bench.REF_LIMITS["facets"] and o.n_points <= bench.REF_LIMITS["points"]


def test_evaluation_sample_converts_to_fits(tmp_path, monkeypatch):
    import bench

    p = bench.make_input(str(tmp_path), "c2")
    monkeypatch.setattr(os, "cpu_count", lambda: 2)
    v, cores, done, dt = bench.cpu_eval_sample(p, 0.1, 1, 51)
    assert cores == 2 and done == 2 and dt > 0
    # two processes, one evaluation each: fits/s = cores / (51 t_eval)
    assert 0 < v < cores / (51 * dt) * 4
