"""FP64 GPU form vs the CPU oracle, through the C ABI (libps_b200.so).

Both FP64 forms are held to the same bars: PS_FORM_FP64 (the reference's
operation order) and PS_FORM_FAST (rearranged, fused; rounding-level
differences).

Tolerances: one model evaluation (the reference's mrqcof) agrees
to 1e-11 relative (normwise for alpha, beta and the Jacobian rows) -- the
only differences are last-ulp libm results (exp, sin, cos, pow(x,2) = x*x);
whole fits and scans agree to 1e-9 relative in chi2/rms, except on periods
whose LM trajectory is chaotic, i.e. where the reference itself changes by
more than that under a last-ulp perturbation (rebuilt with FMA contraction,
or the bit-identical restatement rebuilt with FMA and/or x*x for pow(x,2));
there the GPU value must lie within ten times the largest such spread.  Dark-facet percentages agree
to 1e-6 (absolute) and the best-period ranking is identical.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_path

pytestmark = pytest.mark.gpu

EVAL_TOL = 1e-11
FIT_TOL = 1e-9


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.linalg.norm(b.ravel()), 1e-300)
    return float(np.linalg.norm((a - b).ravel()) / den)


FORMS = ["fp64", "fast"]


def _form(native, form):
    return {"fp64": native.PS_FORM_FP64, "fast": native.PS_FORM_FAST}[form]


def _pair(native, oracle_lib, name, form="fp64"):
    path = golden_path(name)
    o = oracle_lib.Oracle(path)
    conw_r = o.conw_r
    o.set_conw_r(conw_r)
    g = native.PeriodSearch(path, form=_form(native, form))
    g.set_conw_r(conw_r)
    return g, o


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", ["tiny", "tiny_rel", "c1"])
def test_mrqcof_matches_oracle(native, oracle_lib, name, form):
    g, o = _pair(native, oracle_lib, name, form)
    rng = np.random.default_rng(5)
    for n, pole in ((1, 1), (2, 5), (o.n_periods, 9)):
        a = o.initial_parameters(o.freq(n), pole)
        for trial in range(2):
            if trial:
                a = a + rng.normal(0, 1e-3, a.shape) * (np.abs(a) + 0.1) * (np.array(o.array("ia")) > 0)
            al_o, be_o, x_o = o.mrqcof(a)
            al_g, be_g, x_g = g.mrqcof(a)
            assert abs(x_g - x_o) <= EVAL_TOL * abs(x_o), (name, n, pole, x_g, x_o)
            assert _rel(al_g, al_o) <= EVAL_TOL, (name, n, pole, _rel(al_g, al_o))
            assert _rel(be_g, be_o) <= EVAL_TOL, (name, n, pole, _rel(be_g, be_o))
            y_o, J_o = o.model(a)
            y_g, J_g = g.model(a)
            assert _rel(y_g, y_o) <= EVAL_TOL
            # row by row: each data point's derivative vector
            for r in range(J_o.shape[0]):
                if np.any(J_o[r]):
                    assert _rel(J_g[r], J_o[r]) <= 1e-10, (name, r)
    g.close()


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", ["tiny", "tiny_rel"])
def test_fits_match_oracle(native, oracle_lib, name, form):
    g, o = _pair(native, oracle_lib, name, form)
    worst = 0.0
    for n in range(1, o.n_periods + 1):
        f = o.freq(n)
        for pole in range(1, 11):
            ro, _ = o.fit(f, pole)
            rg = g.fit(f, pole)
            assert rg["niter"] == int(ro["niter"])
            # a singular damped system freezes the fit in both (gauss_errc.c:45-50,
            # mrqmin.c:61); all-relative inputs with free phase parameters do that
            assert rg["status"] == int(ro["status"])
            e = abs(rg["chisq"] - ro["chisq"]) / abs(ro["chisq"])
            worst = max(worst, e)
            assert e <= FIT_TOL, (name, n, pole, rg["chisq"], ro["chisq"])
            assert abs(rg["dev"] - ro["dev"]) <= FIT_TOL * abs(ro["dev"])
            assert abs(rg["totarea"] - ro["totarea"]) <= 1e-9 * abs(ro["totarea"])
            assert abs(rg["dark"] - ro["dark"]) <= 1e-6 * max(abs(ro["totarea"]), 1.0)
            assert abs(rg["lambda_deg"] - ro["lambda_deg"]) <= 1e-6
            assert abs(rg["beta_deg"] - ro["beta_deg"]) <= 1e-6
    g.close()


def _read_full(path):
    import pso

    return pso.read_full(path)


PERTURBED = ("fma_out.full", "var_sq.full", "var_fma.full", "var_fmasq.full")


def perturbed_records(name, files=PERTURBED):
    """Records of the reference's last-ulp perturbations (its FMA rebuild and
    the restatement's perturbed builds, tests/golden/make_golden.py)."""
    paths = [f if os.path.isabs(f) else os.path.join(GOLDEN, name, f) for f in files]
    return [_read_full(p) for p in paths if os.path.exists(p)]


def perturbation_spread(name, ref, files=PERTURBED):
    """Largest change per period among last-ulp perturbations of the
    reference: relative for chi2, in degrees for the pole angles, which a flat
    chi2 valley lets move further than chi2 does."""
    spread = np.zeros(len(ref), dtype=[("chi2", "f8"), ("lambda_deg", "f8"), ("beta_deg", "f8")])
    for x in perturbed_records(name, files):
        spread["chi2"] = np.maximum(spread["chi2"], np.abs(x["chi2"] - ref["chi2"]) / np.abs(ref["chi2"]))
        for key in ("lambda_deg", "beta_deg"):
            spread[key] = np.maximum(spread[key], np.abs(x[key] - ref[key]))
    return spread


def _top(r, k):
    return list(np.argsort(r["chi2"], kind="stable")[:k])


def check_records(gpu, ref, spread, label, perturbed=()):
    """Per-period parity with the chaotic-period triage, plus the ranking:
    top-1/10/20 identical, except at a K where the reference's own last-ulp
    perturbations (`perturbed` records) already reorder its top K -- there the
    ranking is itself chaotic and only the per-period bar applies."""
    assert gpu.shape == ref.shape
    n = len(ref)
    cs = spread["chi2"]
    chaotic = cs > FIT_TOL
    err = np.abs(gpu["chi2"] - ref["chi2"]) / np.abs(ref["chi2"])
    # A chaotic period's own spread is the largest of a handful of perturbed
    # runs, a small sample of how far its LM path can wander; the median
    # spread of the workload's chaotic periods is the floor of its envelope.
    floor = float(np.median(cs[chaotic])) if chaotic.any() else 0.0
    ok = (err <= FIT_TOL) | (chaotic & (err <= np.maximum(cs, max(floor, FIT_TOL)) * 10))
    bad = np.nonzero(~ok)[0]
    assert len(bad) == 0, (label, [(int(i) + 1, float(err[i]), float(cs[i])) for i in bad[:10]])
    if chaotic.sum() >= 5:
        # and in distribution: the GPU strays from the reference no further
        # than the reference strays from itself under last-ulp perturbations
        assert np.median(err[chaotic]) <= 5 * floor, (label, float(np.median(err[chaotic])), floor)
    calm = ~chaotic & (err <= FIT_TOL)
    # within calm periods every field matches (record 0 col 4 is conw there)
    assert np.all(np.abs(gpu["rms"][calm] - ref["rms"][calm]) <= FIT_TOL * np.abs(ref["rms"][calm]))
    assert np.all(np.abs(gpu["period_h"][calm] - ref["period_h"][calm]) <= 1e-9 * ref["period_h"][calm])
    d = np.abs(gpu["dark_pct"] - ref["dark_pct"])
    d[0] = 0.0
    assert np.all(d[calm] <= 1e-6), (label, float(np.max(d[calm])))
    for key in ("lambda_deg", "beta_deg"):
        # 1e-6 degrees, or ten times what the reference's own perturbations move
        tol = np.maximum(1e-6, 10 * spread[key])
        d = np.abs(gpu[key] - ref[key])
        assert np.all(d[calm] <= tol[calm]), (key, [(int(i) + 1, float(d[i]), float(spread[key][i]))
                                                    for i in np.nonzero(calm & (d > tol))[0][:5]])
    for k in (1, min(10, n), min(20, n)):
        if any(_top(x, k) != _top(ref, k) for x in perturbed):
            print(f"{label}: top-{k} reordered by the reference's own perturbations; not compared")
            continue
        assert _top(gpu, k) == _top(ref, k), (label, k)
    return int(chaotic.sum()), float(err.max())


# the reference's own real inputs (survey photometry), first periods each
REAL = sorted(d for d in os.listdir(GOLDEN) if d.startswith("real_")) if os.path.isdir(GOLDEN) else []


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", ["tiny", "tiny_rel", "c1", "shipped", "tiny_conv", "c1_conv"] + REAL)
def test_scan_matches_reference(native, oracle_lib, name, form):
    ref_full = os.path.join(GOLDEN, name, "ref_out.full")
    if not os.path.exists(ref_full):
        pytest.skip("fixture not generated")
    ref = _read_full(ref_full)
    spread = perturbation_spread(name, ref)
    g = native.PeriodSearch(golden_path(name), form=_form(native, form))
    conw_r = g.precalc()
    recs = g.scan(1, len(ref))
    # the first record's 4th column is conw_r * escl^2 in the reference output
    assert abs(conw_r * g.escl * g.escl - ref["dark_pct"][0]) <= 1e-12 * ref["dark_pct"][0]
    n_chaotic, worst = check_records(recs, ref, spread, name, perturbed_records(name))
    print(f"{name} {form}: {n_chaotic} chaotic periods of {len(ref)}, worst chi2 rel err {worst:.3e}")
    g.close()
