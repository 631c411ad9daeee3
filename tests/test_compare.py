"""The period_search_out comparator (periodsearch_b200/compare.py): the
reference validator's rule (validator/period_search_validator4.cpp:71-109)
and the strict parity rule, on the golden outputs and planted deviations."""
import numpy as np
import pytest

from conftest import golden_path
from periodsearch_b200 import compare


def test_identical_outputs_match_both_rules(tmp_path):
    out = golden_path("c1", "ref_out.txt")
    assert compare.main([out, out, "--rule", "boinc"]) == 0
    assert compare.main([out, out, "--rule", "strict"]) == 0
    full = golden_path("c1", "ref_out.full")
    assert compare.main([out, out, "--full-a", full, "--full-b", full]) == 0


def test_boinc_rule_tolerances(tmp_path):
    a = compare.read_out(golden_path("c1", "ref_out.txt"))
    b = a.copy()
    # chi2: |a-b|/(a+b)/2 <= 0.5 always holds for positive values, so only
    # period and rms can fail; rms 1.6x larger: |0.6|/2.6/2 = 0.115 > 0.1
    b["rms"][3] *= 1.6
    assert not compare.boinc_match(a, b)
    b = a.copy()
    b["rms"][3] *= 1.5  # 0.5/2.5/2 = 0.1: not above the tolerance
    assert compare.boinc_match(a, b)
    b = a.copy()
    b["chi2"][7] *= 100.0
    assert compare.boinc_match(a, b)
    assert not compare.boinc_match(a, a[:-1])
    assert not compare.boinc_match(a[:0], a[:0])


def test_strict_rule_catches_planted_deviations(tmp_path):
    full = compare.read_out(golden_path("c1", "ref_out.full"))
    b = full.copy()
    b["chi2"][5] *= 1 + 3e-9
    rep = compare.strict_report(full, b, 1e-9, printed=False)
    assert not rep["match"] and any("chi2" in f for f in rep["failures"])
    b = full.copy()
    b["chi2"][5] *= 1 + 5e-10
    assert compare.strict_report(full, b, 1e-9, printed=False)["match"]
    # swapping the two best periods' chi2 changes the ranking
    b = full.copy()
    order = np.argsort(full["chi2"], kind="stable")
    b["chi2"][order[0]], b["chi2"][order[1]] = full["chi2"][order[1]], full["chi2"][order[0]]
    rep = compare.strict_report(full, b, 1.0, printed=False)
    assert any("ranking" in f for f in rep["failures"])


def test_parse_errors(tmp_path):
    bad = tmp_path / "bad"
    bad.write_text("12.0  0.1  nan 1.0 10 20\n")
    good = golden_path("c1", "ref_out.txt")
    assert compare.main([str(bad), good, "--rule", "boinc"]) == 2
    bad.write_text("12.0  0.1\n")
    assert compare.main([str(bad), good]) == 2


def test_reference_validator_known_answer(tmp_path):
    """The reference's TestValidator case (period_search_pure_cpu_win/
    UnitTest_pure_cpu_win/InnerFunctionsTests.cpp:1059-1095): the AVX and the
    plain CPU builds' records for one period match under the validator rule;
    the strict rule (1e-9 or half a printed digit) tells them apart."""
    a = tmp_path / "avx"
    b = tmp_path / "cpu"
    a.write_text("17.20899774  0.167425  3.307656  1.6   96   59\n")
    b.write_text("17.20899838  0.167423  3.307587  1.6   96   59\n")
    assert compare.main([str(a), str(b), "--rule", "boinc"]) == 0
    assert compare.main([str(a), str(b), "--rule", "strict"]) == 1
