"""Comparator for period_search_out files.

Two rules:

* ``boinc`` -- the reference project's result validator
  (validator/period_search_validator4.cpp:71-109): the files must have the
  same, non-zero number of records, and for every record the relative
  difference |a - b| / (a + b) / 2 of the period, of the rms and of the chi2
  must not exceed 0.1, 0.1 and 0.5.  A record that does not parse as six
  numbers, or whose period, rms or chi2 is NaN, is a parse error
  (init_result, :51-53).
* ``strict`` -- the parity rule of this project at the printed precision:
  chi2 and rms within a relative tolerance (default 1e-9) or within half a
  unit of the last printed digit, periods within 1e-9 relative or half a
  printed digit, the dark-facet column within 1e-6 or half a printed digit,
  and the same order of the K best periods by chi2 (K = 1, 10, 20); the pole
  angles are reported, not checked.  With the unrounded side files
  (``.full``, the same six columns at full precision) the printed-digit
  floors drop out.

    python -m periodsearch_b200.compare OUT_A OUT_B [--rule boinc|strict]
        [--tol 1e-9] [--full-a A.full --full-b B.full]

Exit status 0 when the files match, 1 when they do not, 2 on a parse error.
"""
from __future__ import annotations

import argparse
import math
import sys

import numpy as np

COLUMNS = ("period_h", "rms", "chi2", "dark_pct", "lambda_deg", "beta_deg")
RECORD = np.dtype([(c, "f8") for c in COLUMNS])
# printed precision of each column ("%.8f  %.6f  %.6f %4.1f %4.0f %4.0f")
PRINT_STEP = (1e-8, 1e-6, 1e-6, 0.1, 1.0, 1.0)


class ParseError(ValueError):
    pass


def read_out(path: str) -> np.ndarray:
    """Records of a period_search_out (or .full) file."""
    rows = []
    with open(path) as f:
        for n, line in enumerate(f, 1):
            if not line.strip():
                continue
            parts = line.split()
            if len(parts) < 6:
                raise ParseError(f"{path}:{n}: {len(parts)} fields")
            try:
                vals = [float(x) for x in parts[:6]]
            except ValueError as e:
                raise ParseError(f"{path}:{n}: {e}") from None
            if any(math.isnan(v) for v in vals[:3]):
                raise ParseError(f"{path}:{n}: NaN period, rms or chi2")
            rows.append(tuple(vals))
    return np.array(rows, dtype=RECORD)


def boinc_match(a: np.ndarray, b: np.ndarray) -> bool:
    """The reference validator's compare_results."""
    if len(a) == 0 or len(b) == 0 or len(a) != len(b):
        return False
    for key, tol in (("period_h", 0.1), ("rms", 0.1), ("chi2", 0.5)):
        x, y = a[key], b[key]
        with np.errstate(divide="ignore", invalid="ignore"):
            d = np.abs((x - y) / (x + y)) / 2
        # a NaN ratio (0/0) never exceeds the tolerance in the reference
        if np.any(d > tol):
            return False
    return True


def strict_report(a: np.ndarray, b: np.ndarray, tol: float = 1e-9, printed: bool = True) -> dict:
    """Per-column worst deviations and the verdict of the strict rule.
    `printed` adds half a unit of each column's last printed digit to the
    tolerance (for period_search_out files; not for .full files)."""
    rep = {"records": (len(a), len(b)), "match": False, "worst": {}, "failures": []}
    if len(a) != len(b) or len(a) == 0:
        rep["failures"].append("record counts differ or are zero")
        return rep
    rel = {"period_h": tol, "rms": tol, "chi2": tol}
    absol = {"dark_pct": 1e-6}
    for i, key in enumerate(COLUMNS):
        x, y = a[key], b[key]
        d = np.abs(x - y)
        if key in ("lambda_deg", "beta_deg"):
            rep["worst"][key] = float(np.max(d))  # reported, not checked: flat chi2 valleys move them
            continue
        floor = 0.5 * PRINT_STEP[i] * (1 + 1e-9) if printed else 0.0
        if key in rel:
            lim = np.maximum(rel[key] * np.abs(y), floor)
            rep["worst"][key] = float(np.max(d / np.maximum(np.abs(y), 1e-300)))
        else:
            lim = np.full(len(y), max(absol[key], floor))
            lim[0] = np.inf  # the first record prints conw_r escl^2 in the dark column
            rep["worst"][key] = float(np.max(d[1:], initial=0.0))
        for j in np.nonzero(d > lim)[0][:5]:
            rep["failures"].append(f"record {j + 1} {key}: {x[j]!r} vs {y[j]!r}")
    for k in (1, min(10, len(a)), min(20, len(a))):
        ra = list(np.argsort(a["chi2"], kind="stable")[:k])
        rb = list(np.argsort(b["chi2"], kind="stable")[:k])
        if ra != rb:
            rep["failures"].append(f"top-{k} ranking differs")
    rep["match"] = not rep["failures"]
    return rep


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("out_a")
    ap.add_argument("out_b")
    ap.add_argument("--rule", choices=("boinc", "strict"), default="strict")
    ap.add_argument("--tol", type=float, default=1e-9, help="relative chi2/rms/period tolerance (strict rule)")
    ap.add_argument("--full-a", help="unrounded side file of OUT_A")
    ap.add_argument("--full-b", help="unrounded side file of OUT_B")
    args = ap.parse_args(argv)
    try:
        a, b = read_out(args.out_a), read_out(args.out_b)
        fa = read_out(args.full_a) if args.full_a else None
        fb = read_out(args.full_b) if args.full_b else None
    except (ParseError, OSError) as e:
        print(f"parse error: {e}", file=sys.stderr)
        return 2
    if args.rule == "boinc":
        ok = boinc_match(a, b)
        print("match" if ok else "no match")
        return 0 if ok else 1
    if fa is not None and fb is not None:
        rep = strict_report(fa, fb, args.tol, printed=False)
    else:
        rep = strict_report(a, b, args.tol, printed=True)
    for line in rep["failures"]:
        print(line)
    print(("match" if rep["match"] else "no match") + f" ({rep['records'][0]} records, worst {rep['worst']})")
    return 0 if rep["match"] else 1


if __name__ == "__main__":
    sys.exit(main())
