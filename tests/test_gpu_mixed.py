"""Mixed-precision form (PS_FORM_MIXED) vs the CPU oracle / the reference.

The model brightness, chi2, beta, the solve and the rotation angle are FP64;
derivatives are FP32 and the shape block of the Jacobian comes from the
tensor cores in split BF16 (~2^-16 relative per product, FP32 accumulation).

What holds, and is asserted:
  * one evaluation: chi2 and y to 1e-11 (FP64 path); alpha, beta and the
    Jacobian to 1e-4 normwise;
  * every fit runs the reference's iteration count.

What does not hold, and is measured instead: per-period chi2 within 1e-6 of
the reference.  Under the reference's stop rule (a fixed 50 iterations for
these inputs) the fits are far from converged -- chi2 still moves by
0.5-15 % between iterations 50 and 100 on c1 -- so the chi2 reached at
iteration 50 depends on the exact LM path, and a ~1e-5 relative Jacobian
error moves it by ~1e-3 (median) and can reorder the best periods.  The
scan test bounds that drift (median below 1e-2) and prints the distribution;
the FP64 forms are the ones held to the parity bar (test_gpu_parity.py).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_path

pytestmark = pytest.mark.gpu

MIX_TOL = 1e-6


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _pair(native, oracle_lib, name):
    path = golden_path(name)
    o = oracle_lib.Oracle(path)
    o.set_conw_r(o.conw_r)
    g = native.PeriodSearch(path, form=native.PS_FORM_MIXED)
    g.set_conw_r(o.conw_r)
    return g, o


@pytest.mark.parametrize("name", ["tiny", "tiny_rel", "c1"])
def test_mixed_evaluation(native, oracle_lib, name):
    g, o = _pair(native, oracle_lib, name)
    for n, pole in ((1, 1), (2, 5), (o.n_periods, 9)):
        a = o.initial_parameters(o.freq(n), pole)
        al_o, be_o, x_o = o.mrqcof(a)
        al_g, be_g, x_g = g.mrqcof(a)
        assert abs(x_g - x_o) <= 1e-11 * abs(x_o), (name, x_g, x_o)
        assert _rel(be_g, be_o) <= 1e-4, (name, _rel(be_g, be_o))
        assert _rel(al_g, al_o) <= 1e-4, (name, _rel(al_g, al_o))
        y_o, J_o = o.model(a)
        y_g, J_g = g.model(a)
        assert _rel(y_g, y_o) <= 1e-11
        assert _rel(J_g, J_o) <= 1e-4, (name, _rel(J_g, J_o))
    g.close()


@pytest.mark.parametrize("name", ["tiny", "c1"])
def test_mixed_fits_run_the_reference_iterations(native, oracle_lib, name):
    g, o = _pair(native, oracle_lib, name)
    errs = []
    for n in (1, 2, o.n_periods):
        f = o.freq(n)
        for pole in range(1, 11):
            ro, _ = o.fit(f, pole)
            rg = g.fit(f, pole)
            assert rg["niter"] == int(ro["niter"])
            assert np.isfinite(rg["chisq"])
            errs.append(abs(rg["chisq"] - ro["chisq"]) / abs(ro["chisq"]))
    errs = np.array(errs)
    print(f"{name} mixed fits: chi2 rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    g.close()


@pytest.mark.parametrize("name", ["tiny", "c1", "shipped"])
def test_mixed_scan_drift(native, oracle_lib, name):
    import pso

    ref = pso.read_full(os.path.join(GOLDEN, name, "ref_out.full"))
    g = native.PeriodSearch(golden_path(name), form=native.PS_FORM_MIXED)
    conw_r = g.precalc()
    assert abs(conw_r * g.escl * g.escl - ref["dark_pct"][0]) <= 1e-12 * ref["dark_pct"][0]
    recs = g.scan(1, len(ref))
    assert np.all(np.isfinite(recs["chi2"]))
    err = np.abs(recs["chi2"] - ref["chi2"]) / np.abs(ref["chi2"])
    best_same = int(np.argmin(recs["chi2"])) == int(np.argmin(ref["chi2"]))
    print(f"{name} mixed scan: chi2 rel err median {np.median(err):.2e} p90 {np.quantile(err, 0.9):.2e} "
          f"max {err.max():.2e}, best period identical: {best_same}")
    assert np.median(err) <= 1e-2
    g.close()


_WAIT_CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
import periodsearch_b200 as ps
g = ps.PeriodSearch(sys.argv[2], form=ps.PS_FORM_MIXED)
g.set_conw_r(g.conw_r)
try:
    g.scan(1, 3)
    print("NO_ERROR")
except ps.PeriodSearchError as e:
    print("CODE", e.code)
g.close()
cs = [ps.PeriodSearch(sys.argv[2], form=ps.PS_FORM_MIXED) for _ in range(2)]
for c in cs:
    c.set_conw_r(c.conw_r)
b = ps.PeriodSearchBatch(cs)
try:
    b.scan([1, 1], [2, 3])
    print("BATCH_NO_ERROR")
except ps.PeriodSearchError as e:
    print("BATCH_CODE", e.code)
b.close()
for c in cs:
    c.close()
h = ps.PeriodSearch(sys.argv[2], form=ps.PS_FORM_FP64)
h.set_conw_r(h.conw_r)
rec = h.scan(1, 3)
print("AFTER", int(all(rec["chi2"] > 0)))
"""


def test_bounded_wait_gives_up_and_reports(native, tmp_path):
    """The tensor-core waits of the mixed kernel are bounded.  With the limit
    set to zero polls (PS_B200_MAX_POLLS=0) every such wait gives up at
    once: the kernel drains its own MMAs, frees its TMEM and returns, the scan
    reports PS_ERR_DEVICE_LOOP (a single scan and a batched one), and the
    GPU context stays usable (an FP64 scan in the same process afterwards
    succeeds)."""
    import subprocess
    import sys

    from conftest import REPO

    script = tmp_path / "child.py"
    script.write_text(_WAIT_CHILD)
    env = dict(os.environ, PS_B200_MAX_POLLS="0")
    r = subprocess.run([sys.executable, str(script), REPO, golden_path("tiny")], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "\nCODE %d" % native.PS_ERR_DEVICE_LOOP in "\n" + r.stdout, r.stdout
    assert "BATCH_CODE %d" % native.PS_ERR_DEVICE_LOOP in r.stdout, r.stdout
    assert "AFTER 1" in r.stdout, r.stdout
