"""The drop-in executable periodsearch_b200/period_search_b200: the
reference's file contract (period_search_in -> period_search_out, in the
reference's 6-column format), checkpoint/resume through period_search_state
(the CUDA application's "nlines newConw conw_r" form, the CPU application's
bare "nlines", which re-runs the convexity pre-pass, and the five-field
"nlines newConw conw_r sum_dark_facet ntestperiods" form of the pure-CPU and
OpenCL applications, period_search_pure_cpu_win/period_search/
period_search_BOINC.cpp:91,257, whose first three fields are read and whose
interrupted pre-pass is run again from the start), and the reference's exit
codes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden_path

EXE = os.path.join(REPO, "periodsearch_b200", "period_search_b200")


def _lines_close(got, want):
    """Printed records agree: same columns, numbers equal to the printed
    precision except in the last printed digit (rounding of values that
    differ by ~1e-9 relative can straddle a printed digit)."""
    assert len(got) == len(want)
    for g, w in zip(got, want):
        gv = [float(x) for x in g.split()]
        wv = [float(x) for x in w.split()]
        assert len(gv) == len(wv) == 6
        for a, b, q in zip(gv, wv, (1e-8, 1e-6, 1e-6, 0.1, 1.0, 1.0)):
            assert abs(a - b) <= q * 1.01, (g, w)


def _run(d, *args):
    return subprocess.run([EXE, "--dir", str(d), *args], capture_output=True, text=True, timeout=600)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "c1"])
def test_executable_matches_reference_output(native, tmp_path, name):
    shutil.copy(golden_path(name), tmp_path / "period_search_in")
    r = _run(tmp_path)
    assert r.returncode == 0, r.stderr
    got = (tmp_path / "period_search_out").read_text().splitlines()
    want = open(golden_path(name, "ref_out.txt")).read().splitlines()
    _lines_close(got, want)
    n = len(want)
    assert (tmp_path / "period_search_state").read_text().split()[0] == str(n)


@pytest.mark.gpu
@pytest.mark.parametrize("state_form", ["cuda", "cpu", "five", "five_prepass"])
def test_executable_resumes_from_checkpoint(native, tmp_path, state_form):
    shutil.copy(golden_path("tiny"), tmp_path / "period_search_in")
    full = tmp_path / "full"
    full.mkdir()
    shutil.copy(golden_path("tiny"), full / "period_search_in")
    assert _run(full).returncode == 0
    whole = (full / "period_search_out").read_text().splitlines(True)
    state = (full / "period_search_state").read_text().split()
    # interrupted after two periods (or, five_prepass, during the pre-pass)
    done = 0 if state_form == "five_prepass" else 2
    (tmp_path / "period_search_out").write_text("".join(whole[:done]))
    if state_form == "cuda":
        (tmp_path / "period_search_state").write_text("2 1 %s" % state[2])
    elif state_form == "five":
        (tmp_path / "period_search_state").write_text("2 1 %s 3.5 10" % state[2])
    elif state_form == "five_prepass":
        (tmp_path / "period_search_state").write_text("0 0 %s 1.25 3" % state[2])
    else:
        (tmp_path / "period_search_state").write_text("2")
    r = _run(tmp_path, "--chunk", "1")
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "period_search_out").read_text().splitlines(True) == whole


def test_executable_exit_codes(native, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("executable not built")
    r = _run(tmp_path)  # no input file
    assert r.returncode == 255  # exit(-1)
    (tmp_path / "period_search_in").write_text("90 0.5 100 1\n0\n")
    r = _run(tmp_path)
    assert r.returncode == 2


@pytest.mark.gpu
def test_sharded_scan_merges_to_the_unsharded_output(native, tmp_path):
    """Two shards run one after the other on one GPU (--shard 0/2, 1/2, in
    blocks of 7 periods), one of them interrupted and resumed, then --merge 2:
    period_search_out and period_search_state equal the unsharded run's
    byte for byte."""
    full = tmp_path / "full"
    full.mkdir()
    shutil.copy(golden_path("c1"), full / "period_search_in")
    r = _run(full, "--chunk", "7")
    assert r.returncode == 0, r.stderr
    d = tmp_path / "sharded"
    d.mkdir()
    shutil.copy(golden_path("c1"), d / "period_search_in")
    for k in (0, 1):
        r = _run(d, "--shard", f"{k}/2", "--chunk", "7")
        assert r.returncode == 0, r.stderr
    # incomplete shards are refused: drop shard 1's last block and its state
    s1 = d / "period_search_out.shard_1_of_2"
    st1 = d / "period_search_state.shard_1_of_2"
    whole1 = s1.read_text()
    lines = whole1.splitlines(True)
    s1.write_text("".join(lines[:-7] if len(lines) > 8 else lines))
    done, newc, cw = st1.read_text().split()
    st1.write_text("%d %s %s" % (int(done) - 1, newc, cw))
    assert _run(d, "--merge", "2").returncode == 2
    # resume the interrupted shard, then merge
    r = _run(d, "--shard", "1/2", "--chunk", "7")
    assert r.returncode == 0, r.stderr
    assert s1.read_text() == whole1
    r = _run(d, "--merge", "2")
    assert r.returncode == 0, r.stderr
    assert (d / "period_search_out").read_text() == (full / "period_search_out").read_text()
    assert (d / "period_search_state").read_text() == (full / "period_search_state").read_text()
