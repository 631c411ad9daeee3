"""Host-side checks of the product library that need no GPU: the C ABI
library loads and exports every declared symbol, the host setup
(parse + geometry, period_search_BOINC.cpp:277-802) equals the oracle's bit
for bit, errors come back as status codes, and records format exactly like
the reference prints them."""
import os
import re

import numpy as np
import pytest

from conftest import REPO, golden_path

NAMES = ["tiny", "tiny_rel", "c1", "shipped"]


def test_library_exports_every_declared_symbol(native):
    header = open(os.path.join(REPO, "include", "period_search_b200.h")).read()
    declared = set(re.findall(r"\b(ps_[a-z_0-9]+)\s*\(", header))
    assert declared == set(native.EXPORTS)
    lib = native.load_library()
    for name in declared:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("name", NAMES)
def test_host_setup_bitexact_vs_oracle(native, oracle_lib, name):
    path = golden_path(name)
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    o = oracle_lib.Oracle(path)
    o.set_conw_r(o.conw_r)
    h = native.PeriodSearch(path, host_only=True)
    assert h.escl == o.escl and h.n_periods == o.n_periods
    assert (h.numfac, h.ncoef, h.ma, h.mfit) == (o.numfac, o.ncoef, o.ma, o.mfit)
    assert h.freq_start == o.dbls[2] and h.freq_step == o.dbls[4]
    for arr in ("nor", "darea", "dsph", "cg_first", "ia", "tim", "ee", "ee0", "at", "af", "ifp",
                "brightness", "sig", "weight"):
        a, b = o.array(arr), h.array(arr)
        assert a.shape == b.shape and np.array_equal(a, b), arr
    h.close()
    # a second asteroid on the same facet grid takes the grid tables and the
    # grid half of the ellipsoid fit from the per-process cache: same bits
    h2 = native.PeriodSearch(path, host_only=True)
    for arr in ("nor", "dsph", "cg_first"):
        assert np.array_equal(o.array(arr), h2.array(arr)), arr
    h2.close()


def test_errors_are_status_codes(native, tmp_path):
    with pytest.raises(native.PeriodSearchError) as e:
        native.PeriodSearch(str(tmp_path / "missing"), host_only=True)
    assert e.value.code == native.PS_ERR_IO
    bad = tmp_path / "period_search_in"
    bad.write_text("90 0.5 100 1\n0\n0\n0.1\n12 12\n6\n")
    with pytest.raises(native.PeriodSearchError) as e:
        native.PeriodSearch(str(bad), host_only=True)
    assert e.value.code == native.PS_ERR_LIMIT
    h = native.PeriodSearch(golden_path("tiny"), host_only=True)
    lib = native.load_library()
    assert lib.ps_precalc(h._h, None) == native.PS_ERR_ARG
    h.close()


def test_format_record_matches_reference_lines(native, oracle_lib):
    for name in ("tiny", "shipped"):
        full = golden_path(name, "ref_out.full")
        if not os.path.exists(full):
            continue
        recs = oracle_lib.read_full(full)
        lines = open(golden_path(name, "ref_out.txt")).read().splitlines(True)
        for i, r in enumerate(recs):
            # the .full file already carries conw_r*escl^2 in column 4 of line 1
            assert native.format_record(tuple(r)) == lines[i]
