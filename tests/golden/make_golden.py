"""Regenerate the golden fixtures under tests/golden/ (run in the build
container, where the reference sources exist; the fixtures are committed so
that tests never need /root/reference at run time).

    python tests/golden/make_golden.py [names...]

For every workload it writes <name>/period_search_in and the records of the
reference application itself, compiled in place from its own sources by
oracle/Makefile (`make -C oracle ref`):

  ref_out.txt   the reference's printed output (period_search_out)
  ref_out.full  the same six values at %.17g (side file of the stub MFILE)
  fma_out.full  the same source rebuilt with FMA contraction; a period whose
                chi2 differs between the two builds is "chaotic" (its LM
                trajectory amplifies last-ulp differences)
  var_*.full    the oracle restatement (bit-identical to the reference build)
                rebuilt with other last-ulp perturbations -- pow(x,2) -> x*x
                (sq), FMA contraction (fma), both (fmasq) -- at the
                reference's conw_r; together with fma_out.full they define the
                chaotic periods: those that any of these perturbations moves

Long scans are split across host cores the way the reference allows it:
each slice keeps P_start (so the convexity pre-pass sees the same first ten
periods), trims P_end so that the scan stops at the slice end, and starts at
the slice start through period_search_state (period_search_BOINC.cpp:237-251).

Inputs:
  shipped   the reference's own period_search/period_search_in (+ its shipped
            period_search_out as `shipped_out.txt`), first 12 periods
  tiny, tiny_rel, c1   seeded synthetic asteroids (periodsearch_b200.synth)
  tiny_conv, c1_conv   the same with the per-fit convergence stop rule
                       (stop_condition < 1, n_iter_min = 5)
  unit      golden arrays of the reference's unit tests
            (period_search_pure_cpu_win/UnitTest_pure_cpu_win/arrangers.cpp),
            dumped to unit.json through a small C++ harness
  c2        the benchmarked production size: 20 trial periods spread over
            2-100 h, from the reference application (+ FMA build, variants)
  c4_shaped three large asteroids of the uneven batch (up to 4 793 points,
            convergence rule) and c5 (one period of the 20 000-point,
            2 048-facet workload): beyond the reference application's static
            arrays, so from the restatement (-O3, fma, sq builds); their
            inputs are regenerated by periodsearch_b200.synth at test time
            and checked against the sha256 stored in meta.json

  real      the first 20 trial periods (pre-pass included) of six of the
            reference's 100 real inputs (period_search/input_period_search),
            from the reference application and its perturbed builds

Not in the default set (minutes of CPU each): real, c2, c4_shaped, c5.
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

REF_ROOT = os.environ.get("PS_REFERENCE_DIR", "/root/reference")
REF_EXE = os.path.join(REPO, "oracle", "_ref", "period_search_ref")
REF_FMA = os.path.join(REPO, "oracle", "_ref", "period_search_ref_fma")


def _header_values(text):
    first = text.split("\n", 1)[0].split()
    return float(first[0]), float(first[1]), float(first[2]), int(first[3])


def _jd_span(text):
    lines = text.splitlines()
    i = 15  # after the 14 header lines and the lightcurve count
    nlc = int(lines[14].split()[0])
    jd = []
    for _ in range(nlc):
        n = int(lines[i].split()[0])
        for k in range(n):
            jd.append(float(lines[i + 1 + k].split()[0]))
        i += n + 1
    return min(jd), max(jd)


def _n_per(p_start, coef, p_end, jd_min, jd_max):
    f_start = 1 / p_start
    f_end = 1 / p_end
    f_step = 0.5 / (jd_max - jd_min) / 24 * coef
    return int((f_start - f_end) / f_step) + 1


def _slice_text(text, n_end):
    """Same input with P_end moved so that the scan has exactly n_end periods."""
    p_start, coef, p_end, ia = _header_values(text)
    jd_min, jd_max = _jd_span(text)
    f_start = 1 / p_start
    f_step = 0.5 / (jd_max - jd_min) / 24 * coef
    for frac in (0.5, 0.3, 0.7, 0.1, 0.9):
        pe = float("%.12f" % (1 / (f_start - (n_end - 1 + frac) * f_step)))
        if _n_per(p_start, coef, pe, jd_min, jd_max) == n_end:
            rest = text.split("\n", 1)
            tail = rest[0].split(None, 4)[4] if len(rest[0].split(None, 4)) > 4 else ""
            return "%.10f %g %.12f %d %s\n%s" % (p_start, coef, pe, ia, tail, rest[1])
    raise RuntimeError("cannot place P_end for %d periods" % n_end)


def _run_slice(exe, text, n_from, n_to):
    d = tempfile.mkdtemp(prefix="psgold")
    try:
        with open(os.path.join(d, "period_search_in"), "w") as f:
            f.write(_slice_text(text, n_to))
        if n_from > 1:
            with open(os.path.join(d, "period_search_state"), "w") as f:
                f.write("%d" % (n_from - 1))
        subprocess.run([exe], cwd=d, check=True, stdout=subprocess.DEVNULL)
        txt = open(os.path.join(d, "period_search_out")).read()
        full = open(os.path.join(d, "period_search_out.full")).read()
        return txt, full
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_reference(exe, text, n_periods, workers):
    per = max(1, -(-n_periods // workers))
    slices = [(a, min(a + per - 1, n_periods)) for a in range(1, n_periods + 1, per)]
    with cf.ProcessPoolExecutor(max_workers=workers) as ex:
        outs = list(ex.map(_run_slice, [exe] * len(slices), [text] * len(slices),
                           [s[0] for s in slices], [s[1] for s in slices]))
    return "".join(o[0] for o in outs), "".join(o[1] for o in outs)


def _run_variant_slice(exe, text, n_from, n_to, conw_r):
    d = tempfile.mkdtemp(prefix="psvar")
    try:
        open(os.path.join(d, "period_search_in"), "w").write(text)
        subprocess.run([exe, d, str(n_from), str(n_to), "%.17g" % conw_r], check=True, stdout=subprocess.DEVNULL)
        return open(os.path.join(d, "period_search_out.full")).read()
    finally:
        shutil.rmtree(d, ignore_errors=True)


def make_variants(name, workers):
    import math

    import pso

    d = os.path.join(HERE, name)
    text = open(os.path.join(d, "period_search_in")).read()
    ref = pso.read_full(os.path.join(d, "ref_out.full"))
    o = pso.Oracle(os.path.join(d, "period_search_in"))
    k = round(math.log2(ref["dark_pct"][0] / (o.conw_r * o.escl * o.escl)))
    conw_r = o.conw_r * 2.0**k
    n = len(ref)
    per = max(1, -(-n // workers))
    slices = [(a, min(a + per - 1, n)) for a in range(1, n + 1, per)]
    for var in ("sq", "fma", "fmasq"):
        exe = os.path.join(REPO, "oracle", "ps_oracle_" + var)
        with cf.ProcessPoolExecutor(max_workers=workers) as ex:
            outs = list(ex.map(_run_variant_slice, [exe] * len(slices), [text] * len(slices),
                               [s[0] for s in slices], [s[1] for s in slices], [conw_r] * len(slices)))
        open(os.path.join(d, "var_%s.full" % var), "w").write("".join(outs))
    print(name, "variants written", flush=True)


def make_workload(name, text, n_periods, workers):
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "period_search_in"), "w") as f:
        f.write(text)
    txt, full = run_reference(REF_EXE, text, n_periods, workers)
    open(os.path.join(d, "ref_out.txt"), "w").write(txt)
    open(os.path.join(d, "ref_out.full"), "w").write(full)
    _, full_fma = run_reference(REF_FMA, text, n_periods, workers)
    open(os.path.join(d, "fma_out.full"), "w").write(full_fma)
    print(name, n_periods, "periods written", flush=True)


UNIT_HARNESS = r"""
#include <cstdio>
#include "arrangers.hpp"
#include "constants.h"
#include "globals.h"
int Lmax, Mmax, Niter, Lastcall, Ncoef, Numfac, Lcurves, Nphpar, Deallocate, n_iter;
int Lpoints[MAX_LC + 1], Inrel[MAX_LC + 1];
double Alamda, Alamda_incr, Alamda_start, Ochisq, Chisq, _Chisq, Phi_0, Scale, _scale;
double Blmat[4][4], _blmat[4][4], Dblm[3][4][4], _dblm[3][4][4];
double Xx1[4], Xx2[4], _xx1[4], _xx2[4];
double tmat[4][4], dtm[4][4][4], _tmat[4][4], _dtm[4][4][4];
double php[N_PHOT_PAR + 1], dphp[N_PHOT_PAR + 1], _dphp[N_PHOT_PAR + 1];
double Sclnw[MAX_LC + 1], Yout[MAX_N_OBS + 1], Weight[MAX_N_OBS + 1];
double Fc[MAX_N_FAC + 1][MAX_LM + 1], Fs[MAX_N_FAC + 1][MAX_LM + 1], Tc[MAX_N_FAC + 1][MAX_LM + 1], Ts[MAX_N_FAC + 1][MAX_LM + 1];
double Dsph[MAX_N_FAC + 1][MAX_N_PAR + 1], _dsph[MAX_N_FAC + 1][MAX_N_PAR + 1];
double Pleg[MAX_N_FAC + 1][MAX_LM + 1][MAX_LM + 1], _pleg[MAX_N_FAC + 1][MAX_LM + 1][MAX_LM + 1];
double Area[MAX_N_FAC + 1], Darea[MAX_N_FAC + 1], Nor[3][MAX_N_FAC + 1], Dg[MAX_N_FAC + 1][MAX_N_PAR + 1];
double _area[MAX_N_FAC + 1], _darea[MAX_N_FAC + 1], _nor[3][MAX_N_FAC + 1], _dg[MAX_N_FAC + 1][MAX_N_PAR + 1];
double Dyda[MAX_N_PAR + 1], _dyda[MAX_N_PAR + 1];
static void arr(const char* name, const double* a, int n, bool last = false) {
  std::printf("\"%s\": [", name);
  for (int i = 0; i < n; i++) std::printf(i ? ", %.17g" : "%.17g", a[i]);
  std::printf("]%s\n", last ? "" : ",");
}
int main() {
  static double t[MAX_N_FAC + 1], f[MAX_N_FAC + 1], at[MAX_N_FAC + 1], af[MAX_N_FAC + 1], cg[MAX_N_PAR + 1];
  static int ifp_rows[MAX_N_FAC + 1][4];
  int* ifp[MAX_N_FAC + 1];
  for (int i = 0; i <= MAX_N_FAC; i++) ifp[i] = ifp_rows[i];
  get_t(t); get_f(f); get_at(at); get_af(af); get_ifp(ifp);
  Lmax = Mmax = 3; Ncoef = 16; Numfac = 288;
  get_cg_first(16, cg); get_pleg(); get_dsph(); get_area(); get_dg();
  std::printf("{\n");
  arr("t", t + 1, 146); arr("f", f + 1, 146); arr("at", at + 1, 288); arr("af", af + 1, 288);
  static double ifpd[288 * 3];
  for (int i = 1; i <= 288; i++) for (int j = 1; j <= 3; j++) ifpd[(i - 1) * 3 + j - 1] = ifp[i][j];
  arr("ifp", ifpd, 288 * 3);
  arr("cg_first", cg + 1, 16);
  static double pl[288 * 16], ds[288 * 16], dg[288 * 16];
  for (int i = 1; i <= 288; i++) {
    for (int l = 0; l <= 3; l++) for (int m = 0; m <= 3; m++) pl[(i - 1) * 16 + l * 4 + m] = _pleg[i][l][m];
    for (int k = 1; k <= 16; k++) ds[(i - 1) * 16 + k - 1] = _dsph[i][k];
  }
  // get_area / get_dg hold zero-based arrays (facet i+1, coefficient k+1)
  for (int i = 0; i < 288; i++) for (int k = 0; k < 16; k++) dg[i * 16 + k] = _dg[i][k];
  arr("pleg", pl, 288 * 16); arr("dsph", ds, 288 * 16); arr("dg", dg, 288 * 16);
  arr("area", _area, 288, true);
  std::printf("}\n");
  return 0;
}
"""


def make_unit():
    src = os.path.join(REF_ROOT, "period_search_pure_cpu_win", "UnitTest_pure_cpu_win")
    d = tempfile.mkdtemp(prefix="psunit")
    try:
        for h in ("stdafx.h", "CppUnitTest.h", "SDKDDKVer.h", "targetver.h"):
            open(os.path.join(d, h), "w").write("")
        open(os.path.join(d, "harness.cpp"), "w").write(UNIT_HARNESS)
        exe = os.path.join(d, "harness")
        subprocess.run(["g++", "-O0", "-w", "-I", d, "-I", src, "-o", exe, os.path.join(d, "harness.cpp"),
                        os.path.join(src, "arrangers.cpp")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
        data = json.loads(out)
        data["_source"] = ("period_search_pure_cpu_win/UnitTest_pure_cpu_win/arrangers.cpp: get_t, get_f, get_at, "
                           "get_af, get_ifp, get_cg_first, get_pleg, get_dsph, get_dg, get_area "
                           "(TestTrifac/TestAreanorm/TestSphfunc/TestEllfit/TestCurv, InnerFunctionsTests.cpp:165-541)")
        json.dump(data, open(os.path.join(HERE, "unit.json"), "w"))
        print("unit.json written", flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


C2_PERIODS = 20  # trial periods of the c2 slice, spread evenly over its 2-100 h range
C4_ASTEROIDS = (7, 42, 180)  # c4 asteroids with the most points: 39 lightcurves / one 3715- / one 4581-point set
C4_PERIODS = 2
C5_PERIOD = 1


def _sha(text):
    import hashlib

    return hashlib.sha256(text.encode()).hexdigest()


def c2_text():
    """The c2 production workload (N 760, lmax 6, nrows 10, 2-100 h) with the
    convexity weight set to the value its pre-pass ends at (conw x 2^5): the
    reference's pre-pass then stops after one round of 100 fits instead of
    six, with the same conw_r (a power-of-two scaling, exact)."""
    from periodsearch_b200 import synth

    lines = synth._c2().text.split("\n")
    assert lines[3].split()[0] == "0.1"
    lines[3] = "3.2\t\t\t\tconvexity weight"
    return "\n".join(lines)


def _one_period(exe, text, n):
    return _run_slice(exe, text, n, n)


def make_c2_spread(workers):
    """c2 at the benchmarked size: C2_PERIODS trial periods spread over the
    whole 2-100 h range, each one run by the reference application itself
    (and its FMA build) as its own slice (P_end trimmed, started through the
    checkpoint file, pre-pass included), plus the restatement's perturbed
    builds at the same conw_r for the chaotic-period triage."""
    import pso

    d = os.path.join(HERE, "c2")
    os.makedirs(d, exist_ok=True)
    text = c2_text()
    open(os.path.join(d, "period_search_in"), "w").write(text)
    o = pso.Oracle(os.path.join(d, "period_search_in"))
    o.set_conw_r(o.conw_r)
    n_total = o.n_periods
    idx = [1 + round(k * (n_total - 1) / (C2_PERIODS - 1)) for k in range(C2_PERIODS)]
    open(os.path.join(d, "periods.txt"), "w").write("".join("%d\n" % n for n in idx))
    for exe, txt_name, full_name in ((REF_EXE, "ref_out.txt", "ref_out.full"), (REF_FMA, None, "fma_out.full")):
        with cf.ProcessPoolExecutor(max_workers=workers) as ex:
            outs = list(ex.map(_one_period, [exe] * len(idx), [text] * len(idx), idx))
        if txt_name:
            open(os.path.join(d, txt_name), "w").write("".join(t for t, _ in outs))
        open(os.path.join(d, full_name), "w").write("".join(f for _, f in outs))
        print("c2", full_name, "written", flush=True)
    ref = pso.read_full(os.path.join(d, "ref_out.full"))
    import math

    o2 = pso.Oracle(os.path.join(d, "period_search_in"))
    k = round(math.log2(ref["dark_pct"][0] / (o2.conw_r * o2.escl * o2.escl)))
    conw_r = o2.conw_r * 2.0**k
    for var in ("sq", "fma", "fmasq"):
        exe = os.path.join(REPO, "oracle", "ps_oracle_" + var)
        with cf.ProcessPoolExecutor(max_workers=workers) as ex:
            outs = list(ex.map(_run_variant_slice, [exe] * len(idx), [text] * len(idx), idx, idx,
                               [conw_r] * len(idx)))
        open(os.path.join(d, "var_%s.full" % var), "w").write("".join(outs))
    print("c2 variants written", flush=True)


def _restatement_records(name, texts, n_from, n_to, conw_rs, workers):
    """Records of the restatement (ps_oracle: -O3, its perturbed builds) for
    inputs beyond the reference application's static arrays."""
    d = os.path.join(HERE, name)
    for var, exe in (("oracle_out", os.path.join(REPO, "oracle", "ps_oracle")),
                     ("var_fma", os.path.join(REPO, "oracle", "ps_oracle_fma")),
                     ("var_sq", os.path.join(REPO, "oracle", "ps_oracle_sq"))):
        with cf.ProcessPoolExecutor(max_workers=workers) as ex:
            outs = list(ex.map(_run_variant_slice, [exe] * len(texts), texts, n_from, n_to, conw_rs))
        yield var, outs


def make_c4_shaped(workers):
    """Three c4 asteroids (the uneven batch's largest shapes: up to 4 793
    points, one sparse set of 4 581 points, or 39 lightcurves; lmax 6,
    nrows 10, the per-fit convergence rule), C4_PERIODS trial periods each at
    the pre-pass start value conw/escl^2 as the batch benchmark runs them.
    The reference application holds at most 1 000 points per lightcurve
    (constants.h POINTS_MAX), so the records come from the restatement."""
    import pso
    from periodsearch_b200 import synth

    d = os.path.join(HERE, "c4_shaped")
    os.makedirs(d, exist_ok=True)
    texts, conws, meta = [], [], {"asteroids": [], "periods": C4_PERIODS}
    for i in C4_ASTEROIDS:
        w, _ = synth.c4_asteroid(i)
        tmp = tempfile.mkdtemp(prefix="psc4g")
        o = pso.Oracle(synth.write_input(w, tmp))
        texts.append(w.text)
        conws.append(o.conw_r)
        meta["asteroids"].append({"index": i, "sha256": _sha(w.text), "n_points": w.n_points, "conw_r": o.conw_r})
        shutil.rmtree(tmp, ignore_errors=True)
    for var, outs in _restatement_records("c4_shaped", texts, [1] * len(texts), [C4_PERIODS] * len(texts), conws,
                                          workers):
        for i, out in zip(C4_ASTEROIDS, outs):
            open(os.path.join(d, "a%03d_%s.full" % (i, var)), "w").write(out)
    json.dump(meta, open(os.path.join(d, "meta.json"), "w"), indent=1)
    print("c4_shaped written", flush=True)


def c5_workload():
    from periodsearch_b200 import synth

    return synth.make_workload("c5_lmax8_n20000_f2048", 5, dense_lcs=40, dense_pts=100, sparse_pts=16000, years=10,
                               true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2000)


def make_c5(workers):
    """One trial period (10 whole fits) of the c5 workload at full size
    (N 20 000, lmax 8, 2 048 facets) from the restatement and its perturbed
    builds, at the pre-pass start value conw/escl^2 (the benchmark skips the
    pre-pass there too); 2 048 facets exceed the reference application's
    MAX_N_FAC."""
    import pso

    d = os.path.join(HERE, "c5")
    os.makedirs(d, exist_ok=True)
    from periodsearch_b200 import synth

    w = c5_workload()
    tmp = tempfile.mkdtemp(prefix="psc5g")
    o = pso.Oracle(synth.write_input(w, tmp))
    meta = {"sha256": _sha(w.text), "conw_r": o.conw_r, "period": C5_PERIOD}
    shutil.rmtree(tmp, ignore_errors=True)
    jobs = []
    for var in ("ps_oracle", "ps_oracle_fma", "ps_oracle_sq"):
        jobs.append((os.path.join(REPO, "oracle", var), w.text, C5_PERIOD, C5_PERIOD, meta["conw_r"]))
    with cf.ProcessPoolExecutor(max_workers=min(workers, 3)) as ex:
        outs = list(ex.map(_run_variant_slice, *zip(*jobs)))
    for name, out in zip(("oracle_out", "var_fma", "var_sq"), outs):
        open(os.path.join(d, name + ".full"), "w").write(out)
    json.dump(meta, open(os.path.join(d, "meta.json"), "w"), indent=1)
    print("c5 written", flush=True)


REAL_PERIODS = 20  # trial periods of each real-data slice (the pre-pass reads the first ten)


def real_inputs():
    """Six of the reference's 100 real inputs (period_search/input_period_search:
    survey photometry, lmax = mmax = 3, nrows = 6), spread over their sizes."""
    d = os.path.join(REF_ROOT, "period_search", "input_period_search")
    files = sorted(os.listdir(d), key=lambda f: (os.path.getsize(os.path.join(d, f)), f))
    pick = [files[i] for i in (0, 20, 40, 60, 80, len(files) - 1)]
    return [(f.split("_")[-1], open(os.path.join(d, f)).read()) for f in pick]


def _make_real_one(ident, text):
    name = "real_" + ident
    # one slice: the pre-pass must see the first ten periods, as a scan of
    # the whole 20-period input does (a slice ending before period ten would
    # run it on fewer)
    make_workload(name, _slice_text(text, REAL_PERIODS), REAL_PERIODS, 1)
    make_variants(name, 1)
    return name


def make_real(workers):
    """The first REAL_PERIODS trial periods of each real input, pre-pass
    included, from the reference application, its FMA build and the
    restatement's perturbed builds; the inputs in parallel."""
    todo = real_inputs()
    with cf.ProcessPoolExecutor(max_workers=min(workers, len(todo))) as ex:
        list(ex.map(_make_real_one, [i for i, _ in todo], [t for _, t in todo]))


def main(names):
    from periodsearch_b200 import synth

    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "all", "variants", "ref"], check=True)
    workers = os.cpu_count() or 4
    if "unit" in names:
        make_unit()
    if "shipped" in names:
        text = open(os.path.join(REF_ROOT, "period_search", "period_search_in")).read()
        d = os.path.join(HERE, "shipped")
        os.makedirs(d, exist_ok=True)
        shutil.copy(os.path.join(REF_ROOT, "period_search", "period_search_out"), os.path.join(d, "shipped_out.txt"))
        make_workload("shipped", _slice_text(text, 12), 12, 1)
    for name, fn, n in (("tiny", synth._tiny, None), ("tiny_rel", synth._tiny_rel, None), ("c1", synth._c1, None)):
        if name in names:
            w = fn()
            make_workload(name, w.text, w.n_periods, workers if w.n_periods > 20 else 1)
    # the per-fit convergence stop rule (stop_condition < 1, n_iter_min;
    # period_search_BOINC.cpp:855-867): tiny, and the first 40 periods of c1
    for name, fn, stop, nmin, keep in (("tiny_conv", synth._tiny, 0.0005, 5, None),
                                       ("c1_conv", synth._c1, 0.0001, 5, 40)):
        if name in names:
            w = fn()
            lines = w.text.split("\n")
            lines[10] = "%g\t\t\t\titeration stop condition" % stop
            lines[11] = "%d\t\t\t\tminimum number of iterations (only if the above value < 1)" % nmin
            text = "\n".join(lines)
            n = w.n_periods
            if keep:
                text = _slice_text(text, keep)
                n = keep
            make_workload(name, text, n, workers if n > 20 else 1)
    for name in ("tiny", "tiny_rel", "c1", "shipped", "tiny_conv", "c1_conv"):
        if name in names or "variants" in names:
            make_variants(name, workers)
    if "real" in names:
        make_real(workers)
    if "c2" in names:
        make_c2_spread(workers)
    if "c4_shaped" in names:
        make_c4_shaped(workers)
    if "c5" in names:
        make_c5(workers)


if __name__ == "__main__":
    main(sys.argv[1:] or ["unit", "shipped", "tiny", "tiny_rel", "c1", "tiny_conv", "c1_conv", "variants"])
