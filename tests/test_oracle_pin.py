"""Pin the CPU oracle (oracle/ps_oracle.c) against the reference.

* records of the reference application compiled in place
  (tests/golden/*/ref_out.full, written by tests/golden/make_golden.py):
  bit-exact, all six values at full precision;
* the reference's own shipped golden output (period_search/period_search_out,
  first 12 trial periods): identical printed lines;
* the golden arrays of the reference's unit tests
  (period_search_pure_cpu_win/UnitTest_pure_cpu_win/arrangers.cpp):
  triangulation, facet normal angles, Legendre/SH tables, initial
  ellipsoid, facet areas and Dg.
"""
import json
import math
import os
import shutil
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, golden_path


def _conw_r_of(o, ref_first_col4):
    # the reference prints conw_r * escl^2 on line 1; conw_r is conw/escl^2
    # doubled k times by the pre-pass (period_search_BOINC.cpp:708-712)
    conw_r0 = o.conw_r
    k = round(math.log2(ref_first_col4 / (conw_r0 * o.escl * o.escl)))
    return conw_r0 * 2.0**k


@pytest.mark.parametrize("name", ["tiny", "tiny_rel"])
def test_oracle_app_bitexact_vs_reference(oracle_lib, name):
    ref = golden_path(name, "ref_out.full")
    if not os.path.exists(ref):
        pytest.skip("fixture missing")
    d = tempfile.mkdtemp()
    try:
        shutil.copy(golden_path(name), os.path.join(d, "period_search_in"))
        assert oracle_lib.run_app(d) == 0
        got = open(os.path.join(d, "period_search_out.full")).read()
        assert got == open(ref).read()
        assert open(os.path.join(d, "period_search_out")).read() == open(golden_path(name, "ref_out.txt")).read()
    finally:
        shutil.rmtree(d, ignore_errors=True)


@pytest.mark.parametrize("name", ["c1", "shipped"])
def test_oracle_slices_bitexact_vs_reference(oracle_lib, name):
    ref_path = golden_path(name, "ref_out.full")
    if not os.path.exists(ref_path):
        pytest.skip("fixture missing")
    ref = oracle_lib.read_full(ref_path)
    o = oracle_lib.Oracle(golden_path(name))
    o.set_conw_r(_conw_r_of(o, ref["dark_pct"][0]))
    n = len(ref)
    for a, b in ((2, 3), (n, n)):
        got = o.scan(a, b)
        for k in got.dtype.names:
            assert np.array_equal(got[k], ref[k][a - 1:b]), (a, b, k)


def test_oracle_matches_shipped_golden_output(oracle_lib):
    shipped = golden_path("shipped", "shipped_out.txt")
    ours = golden_path("shipped", "ref_out.txt")
    if not os.path.exists(shipped):
        pytest.skip("fixture missing")
    a = open(shipped).read().splitlines()[:12]
    b = open(ours).read().splitlines()
    assert a == b


def test_unit_golden_arrays(oracle_lib):
    gold = json.load(open(os.path.join(GOLDEN, "unit.json")))
    # setup of TestEllfit / TestCurv (InnerFunctionsTests.cpp:356-420, 424-541)
    ave = 0.382008772881355651573898057904
    al0 = 0.069555451868686835048549710336
    a, b, c = 1.05, 1.00, 0.95
    rfit = math.sqrt(2 * ave / (0.5 * math.pi * (1 + math.cos(al0))))
    escl = rfit / math.sqrt((a * b + b * c + a * c) / 3) * 0.8
    o = oracle_lib.Oracle.geometry(3, 3, 6, a * escl, b * escl, c * escl)
    assert np.array_equal(o.array("ifp"), np.array(gold["ifp"]))
    # the arrays were produced with MSVC's libm: acos/atan2 agree to a few ulp
    for k in ("at", "af"):
        np.testing.assert_allclose(o.array(k), gold[k], rtol=0, atol=4 * 2.2e-16 * np.pi)
    # entries that are zero up to roundoff differ at the 1e-16 scale, so the
    # absolute tolerance is a few ulp of the array's largest entry
    def close(got, want, rtol):
        want = np.asarray(want, dtype=np.float64).reshape(got.shape)
        np.testing.assert_allclose(got, want, rtol=rtol, atol=8 * 2.2e-16 * np.max(np.abs(want)))

    close(o.array("pleg").reshape(288, 4, 4), gold["pleg"], 8e-15)
    # get_dsph() holds facets 1..146 only (TestSphfunc checks i < ndir = 146)
    close(o.array("dsph").reshape(288, 16)[:145], np.array(gold["dsph"]).reshape(288, 16)[:145], 8e-15)
    close(o.array("cg_first"), gold["cg_first"], 1e-12)
    area, dg = o.curv(np.array(gold["cg_first"]))
    close(area, gold["area"], 1e-12)
    close(dg, gold["dg"], 1e-12)


def test_gauss_errc_solves_and_flags_singular(oracle_lib):
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 22, 55):
        a = rng.normal(size=(n, n)) + n * np.eye(n)
        b = rng.normal(size=n)
        rc, _, x = oracle_lib.gauss_errc(a, b)
        assert rc == 0
        np.testing.assert_allclose(a @ x, b, rtol=1e-10, atol=1e-10)
    a = np.ones((3, 3))
    rc, _, _ = oracle_lib.gauss_errc(a, np.ones(3))
    assert rc == 2
    rc, _, _ = oracle_lib.gauss_errc(np.zeros((4, 4)), np.ones(4))
    assert rc == 2


def test_synthetic_generator_is_seeded():
    from periodsearch_b200 import synth

    a = synth._tiny()
    b = synth._tiny()
    assert a.text == b.text and a.n_periods == 4
    assert open(golden_path("tiny")).read() == a.text
