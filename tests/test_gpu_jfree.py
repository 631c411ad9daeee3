"""Jacobian-free LM fits (ps_fit_jfree) and the final parameters of ps_fit.

ps_fit_jfree runs the reference's LM loop (mrqmin.c:11-110, the stop rule of
period_search_BOINC.cpp:846-920) with every evaluation from the matrix-free
kernels: alpha from mfit Gauss-Newton products, beta and chi2 from the
gradient pass, the solve on the host.  Held to the same bars as the GPU fit
kernels against the oracle (iteration count and status exact, chi2 and rms
to 1e-9, angles to 1e-6), and at the matrix-free configuration's full size
(N = 20 000, 2048 facets, 81 coefficients) compared with the explicit fit of
the fast form on one trial period and timed.
"""
import math
import time

import numpy as np
import pytest

from conftest import golden_path
from periodsearch_b200 import synth

pytestmark = pytest.mark.gpu

FIT_TOL = 1e-9


def _open(native, oracle_lib, path, form):
    o = oracle_lib.Oracle(path)
    o.set_conw_r(o.conw_r)
    g = native.PeriodSearch(path, form=form)
    g.set_conw_r(o.conw_r)
    return g, o


def _check(rg, ro, tag):
    assert rg["niter"] == int(ro["niter"]), tag
    assert rg["status"] == int(ro["status"]), tag
    assert abs(rg["chisq"] - ro["chisq"]) <= FIT_TOL * abs(ro["chisq"]), (tag, rg["chisq"], ro["chisq"])
    assert abs(rg["dev"] - ro["dev"]) <= FIT_TOL * abs(ro["dev"]), tag
    assert abs(rg["totarea"] - ro["totarea"]) <= 1e-9 * abs(ro["totarea"]), tag
    assert abs(rg["lambda_deg"] - ro["lambda_deg"]) <= 1e-6, tag
    assert abs(rg["beta_deg"] - ro["beta_deg"]) <= 1e-6, tag


@pytest.mark.parametrize("name", ["tiny", "tiny_rel"])
def test_jfree_fits_match_oracle(native, oracle_lib, name):
    g, o = _open(native, oracle_lib, golden_path(name), native.PS_FORM_FAST)
    for n in range(1, o.n_periods + 1):
        f = o.freq(n)
        for pole in (1, 4, 7, 10):
            ro, cg_o = o.fit(f, pole)
            rj, cg_j = g.fit_jfree(f, pole, params=True)
            _check(rj, ro, (name, n, pole, "jfree"))
            # a fit frozen by a singular system (status != 0: all-relative data
            # with free phase parameters) leaves those parameters diverged
            if ro["status"] == 0:
                assert np.linalg.norm(cg_j - cg_o) <= 1e-6 * np.linalg.norm(cg_o), (name, n, pole)
    g.close()


@pytest.mark.parametrize("form", ["fp64", "fast", "mixed"])
def test_fit_returns_final_parameters(native, oracle_lib, form):
    """ps_fit's cg_out: the parameters the fit ended at -- the period and
    pole it reports are theirs, and (FP64 forms) they are the oracle's."""
    fid = {"fp64": native.PS_FORM_FP64, "fast": native.PS_FORM_FAST, "mixed": native.PS_FORM_MIXED}[form]
    g, o = _open(native, oracle_lib, golden_path("tiny"), fid)
    C = g.ncoef
    for n, pole in ((1, 3), (o.n_periods, 8)):
        f = o.freq(n)
        r, cg = g.fit(f, pole, params=True)
        assert r["period_d"] == 2 * math.pi / cg[C + 2]
        assert r["lambda_deg"] == (180 / math.pi) * cg[C + 1]
        assert abs(r["beta_deg"] - (90 - (180 / math.pi) * cg[C])) <= 1e-12  # may be one fused op
        if form != "mixed":
            ro, cg_o = o.fit(f, pole)
            assert ro["status"] == 0
            assert np.linalg.norm(cg - cg_o) <= 1e-6 * np.linalg.norm(cg_o), (form, n, pole)
    g.close()


def test_jfree_full_size(native, oracle_lib, tmp_path):
    w = synth.make_workload("large_full", 5, dense_lcs=40, dense_pts=100, sparse_pts=16000, years=10,
                            true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2)
    path = synth.write_input(w, str(tmp_path))
    g, o = _open(native, oracle_lib, path, native.PS_FORM_FAST)
    assert (g.n_points, g.ncoef, g.mfit) == (20000, 81, 87)
    f = o.freq(1)
    t0 = time.perf_counter()
    re = g.fit(f, 2)
    t_explicit = time.perf_counter() - t0
    t0 = time.perf_counter()
    rj = g.fit_jfree(f, 2)
    t_jfree = time.perf_counter() - t0
    d = abs(rj["chisq"] - re["chisq"]) / abs(re["chisq"])
    print(f"N=20000 F=2048 C=81, one fit of {re['niter']} iterations: explicit (one CTA) {t_explicit:.2f} s, "
          f"Jacobian-free (whole GPU) {t_jfree:.2f} s, chi2 {rj['chisq']:.10e} vs {re['chisq']:.10e} ({d:.1e})")
    assert rj["niter"] == re["niter"] and rj["status"] == re["status"]
    assert d <= 1e-6
    g.close()
