"""The library from C: tests/c/scan_client.c, compiled with gcc against
include/period_search_b200.h and linked to the in-tree libps_b200.so, as a C
caller of the reference's period loop would use it."""
import os
import shutil
import subprocess

import pytest

from conftest import REPO, golden_path

LIBDIR = os.path.join(REPO, "periodsearch_b200")


def _build(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    if not os.path.exists(os.path.join(LIBDIR, "libps_b200.so")):
        pytest.skip("library not built")
    exe = tmp_path / "scan_client"
    subprocess.run(["gcc", "-O2", "-std=c99", "-o", str(exe), os.path.join(REPO, "tests", "c", "scan_client.c"),
                    "-I" + os.path.join(REPO, "include"), "-L" + LIBDIR, "-lps_b200", "-Wl,-rpath," + LIBDIR],
                   check=True)
    return exe


def test_c_client_builds(tmp_path):
    assert os.access(_build(tmp_path), os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [0, 2])
def test_c_client_reproduces_reference_output(tmp_path, form):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), golden_path("tiny"), str(form)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = r.stdout.splitlines()
    want = open(golden_path("tiny", "ref_out.txt")).read().splitlines()
    assert len(got) == len(want)
    for g, w in zip(got, want):
        gv, wv = [float(x) for x in g.split()], [float(x) for x in w.split()]
        for a, b, q in zip(gv, wv, (1e-8, 1e-6, 1e-6, 0.1, 1.0, 1.0)):
            assert abs(a - b) <= q * 1.01, (g, w)
