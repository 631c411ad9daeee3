"""Large shapes (the matrix-free configuration's size class): lmax = mmax = 8
(81 shape coefficients, NCB = 88, mfit = 87) on nrows = 16 (2048 facets),
beyond the reference's MAX_N_FAC = 1000 (constants.h:1-11), so the oracle
is the restatement alone (it has no size limits; it is bit-identical to the
reference wherever the reference runs).

* one model evaluation (mrqcof) at the full size, N = 20 000 points (40
  dense lightcurves of 100 points + 16 000 sparse), against the oracle;
* whole fits at a reduced point count (N = 600), both FP64 forms.
"""
import numpy as np
import pytest

from periodsearch_b200 import synth

pytestmark = pytest.mark.gpu

EVAL_TOL = 1e-11
FIT_TOL = 1e-9


def _workload(tmp_path, full):
    if full:
        w = synth.make_workload("large_full", 5, dense_lcs=40, dense_pts=100, sparse_pts=16000, years=10,
                                true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2)
    else:
        w = synth.make_workload("large_small", 5, dense_lcs=4, dense_pts=50, sparse_pts=400, years=10,
                                true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2)
    return synth.write_input(w, str(tmp_path))


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    return _workload(tmp_path_factory.mktemp("large_small"), False)


@pytest.mark.parametrize("form", ["fp64", "fast"])
def test_full_size_evaluation(native, oracle_lib, tmp_path, form):
    path = _workload(tmp_path, True)
    o = oracle_lib.Oracle(path)
    o.set_conw_r(o.conw_r)
    assert (o.n_points, o.ncoef, o.mfit) == (20000, 81, 87)
    g = native.PeriodSearch(path, form={"fp64": native.PS_FORM_FP64, "fast": native.PS_FORM_FAST}[form])
    g.set_conw_r(o.conw_r)
    a = o.initial_parameters(o.freq(1), 3)
    al_o, be_o, x_o = o.mrqcof(a)
    al_g, be_g, x_g = g.mrqcof(a)
    assert abs(x_g - x_o) <= EVAL_TOL * abs(x_o), (x_g, x_o)
    assert _rel(al_g, al_o) <= EVAL_TOL
    assert _rel(be_g, be_o) <= EVAL_TOL
    g.close()


@pytest.mark.parametrize("form", ["fp64", "fast"])
def test_fits_at_lmax8_nrows16(native, oracle_lib, small, form):
    o = oracle_lib.Oracle(small)
    o.set_conw_r(o.conw_r)
    g = native.PeriodSearch(small, form={"fp64": native.PS_FORM_FP64, "fast": native.PS_FORM_FAST}[form])
    g.set_conw_r(o.conw_r)
    for pole in (1, 6):
        ro, _ = o.fit(o.freq(1), pole)
        rg = g.fit(o.freq(1), pole)
        assert rg["niter"] == int(ro["niter"]) and rg["status"] == int(ro["status"])
        e = abs(rg["chisq"] - ro["chisq"]) / abs(ro["chisq"])
        assert e <= FIT_TOL, (pole, rg["chisq"], ro["chisq"])
        assert abs(rg["dark"] - ro["dark"]) <= 1e-6 * max(abs(ro["totarea"]), 1.0)
    g.close()
