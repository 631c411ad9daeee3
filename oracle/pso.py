"""ctypes wrapper of the CPU oracle (oracle/libps_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs as the checker.  The product
package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libps_oracle.so")
EXE = os.path.join(HERE, "ps_oracle")
REF_EXE = os.path.join(HERE, "_ref", "period_search_ref")
REF_FMA_EXE = os.path.join(HERE, "_ref", "period_search_ref_fma")
# where the reference checkout lies (set PS_REFERENCE_DIR to move it)
REF_SRC = os.path.join(os.environ.get("PS_REFERENCE_DIR", "/root/reference"), "period_search")

RECORD_DTYPE = np.dtype(
    [("period_h", "f8"), ("rms", "f8"), ("chi2", "f8"), ("dark_pct", "f8"), ("lambda_deg", "f8"), ("beta_deg", "f8")]
)
_D = ctypes.POINTER(ctypes.c_double)
_lib = None


def build(ref: bool = True) -> None:
    """Compile the restatement; with ref=True also the reference itself when
    its sources are present (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build(ref=False)
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.pso_load.restype = vp
        L.pso_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        L.pso_free.argtypes = [vp]
        L.pso_prepass.argtypes = [vp, _D]
        L.pso_set_conw_r.argtypes = [vp, ctypes.c_double]
        L.pso_n_periods.argtypes = [vp]
        L.pso_scan.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.pso_fit.argtypes = [vp, ctypes.c_double, ctypes.c_int, _D, _D]
        L.pso_mrqcof.restype = ctypes.c_double
        L.pso_mrqcof.argtypes = [vp, _D, _D, _D]
        L.pso_model.argtypes = [vp, _D, _D, _D]
        L.pso_gauss_errc.argtypes = [_D, ctypes.c_int, _D]
        L.pso_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), _D]
        L.pso_get_array.argtypes = [vp, ctypes.c_char_p, _D]
        L.pso_geometry.restype = vp
        L.pso_geometry.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double]
        L.pso_curv.argtypes = [vp, _D, _D, _D]
        L.pso_run_app.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_D)


class Oracle:
    """The restated reference application on one input file."""

    def __init__(self, path: str | None = None, *, handle=None):
        L = lib()
        if handle is None:
            st = ctypes.c_int(0)
            handle = L.pso_load(os.fsencode(path), ctypes.byref(st))
            if not handle:
                raise RuntimeError(f"oracle could not load {path} (status {st.value})")
        self.h = ctypes.c_void_p(handle)
        self.refresh()

    @classmethod
    def geometry(cls, lmax, mmax, nrows, a, b, c):
        h = lib().pso_geometry(lmax, mmax, nrows, a, b, c)
        if not h:
            raise RuntimeError("oracle geometry setup failed")
        return cls(handle=h)

    def refresh(self):
        ints = (ctypes.c_int * 16)()
        dbls = (ctypes.c_double * 16)()
        lib().pso_info(self.h, ints, dbls)
        self.ints = list(ints)
        self.dbls = list(dbls)
        (self.n_points, self.lcurves, self.numfac, self.ncoef, self.ma, self.mfit, self.n_periods) = self.ints[:7]
        self.escl, self.conw_r = self.dbls[0], self.dbls[1]

    def close(self):
        if self.h:
            lib().pso_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prepass(self) -> float:
        v = ctypes.c_double()
        rc = lib().pso_prepass(self.h, ctypes.byref(v))
        if rc:
            raise RuntimeError(f"oracle pre-pass failed ({rc})")
        self.refresh()
        return v.value

    def set_conw_r(self, conw_r: float):
        rc = lib().pso_set_conw_r(self.h, float(conw_r))
        if rc:
            raise RuntimeError(f"oracle setup failed ({rc})")
        self.refresh()

    def scan(self, n_from: int, n_to: int) -> np.ndarray:
        out = np.zeros(n_to - n_from + 1, dtype=RECORD_DTYPE)
        lib().pso_scan(self.h, n_from, n_to, out.ctypes.data_as(ctypes.c_void_p))
        return out

    def fit(self, freq: float, pole: int):
        out = np.zeros(10)
        cg = np.zeros(self.ma)
        lib().pso_fit(self.h, float(freq), int(pole), _p(out), _p(cg))
        keys = ("dev", "dark", "totarea", "period_d", "lambda_deg", "beta_deg", "chisq", "niter", "alamda", "status")
        return dict(zip(keys, out.tolist())), cg

    def mrqcof(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        alpha = np.zeros((self.mfit, self.mfit))
        beta = np.zeros(self.mfit)
        chi2 = lib().pso_mrqcof(self.h, _p(a), _p(alpha), _p(beta))
        return alpha, beta, chi2

    def model(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        y = np.zeros(self.n_points + 3)
        J = np.zeros((self.n_points + 3, self.ma))
        lib().pso_model(self.h, _p(a), _p(y), _p(J))
        return y, J

    def array(self, name: str) -> np.ndarray:
        buf = np.zeros(max(self.numfac, 1) * (max(self.ncoef, 1) + 3) * 16 + 4 * (self.n_points + 3) + 64)
        n = lib().pso_get_array(self.h, name.encode(), _p(buf))
        if n < 0:
            raise KeyError(name)
        return buf[:n].copy()

    def curv(self, cg):
        cg = np.ascontiguousarray(cg, dtype=np.float64)
        area = np.zeros(self.numfac)
        dg = np.zeros((self.numfac, self.ncoef))
        lib().pso_curv(self.h, _p(cg), _p(area), _p(dg))
        return area, dg

    def initial_parameters(self, freq: float, pole: int) -> np.ndarray:
        """cg at the start of fit (freq, pole), period_search_BOINC.cpp:821-844."""
        beta_pole = [0, 0, 0, 0, 60, 60, 60, -60, -60, -60]
        lambda_pole = [0, 90, 180, 270, 60, 180, 300, 60, 180, 300]
        C = self.ncoef
        cg = np.zeros(self.ma)
        cg[:C] = self.array("cg_first")
        deg2rad = np.pi / 180
        cg[C] = deg2rad * (90.0 - beta_pole[pole - 1])
        cg[C + 1] = deg2rad * lambda_pole[pole - 1]
        prd = 1 / freq
        cg[C + 2] = 24 * 2 * np.pi / prd
        cg[C + 3:C + 6] = self.dbls[13:16]
        cg[C + 6] = np.log(self.dbls[12])
        cg[C + 7] = 1.0
        return cg

    def freq(self, n: int) -> float:
        return self.dbls[2] - (n - 1) * self.dbls[4]


def gauss_errc(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).copy()
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    rc = lib().pso_gauss_errc(_p(a), a.shape[0], _p(b))
    return rc, a, b


def run_app(directory: str, n_from: int = 0, n_to: int = 0, conw_r: float = 0.0) -> int:
    return lib().pso_run_app(os.fsencode(directory), n_from, n_to, conw_r)


def read_full(path: str) -> np.ndarray:
    """Read a period_search_out.full side file (six %.17g values a line)."""
    rows = [tuple(float(x) for x in line.split()) for line in open(path) if line.strip()]
    return np.array(rows, dtype=RECORD_DTYPE)
