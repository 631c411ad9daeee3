"""B200-native convex-inversion period scan (Asteroids@home ``period_search``).

Python host mirror of the reference's GPU operator interface
(period_search_cuda/period_search/start_CUDA.h): ``prepare`` (CUDAPrepare:
parse + upload), ``precalc`` (CUDAPrecalc: convexity-weight pre-pass),
``start`` (CUDAStart: the period scan, returning records instead of writing
an MFILE) and ``unprepare`` (CUDAUnprepare), over the C ABI of
``libps_b200.so`` (include/period_search_b200.h).  The object API
(:class:`PeriodSearch`) is the same calls on an explicit context.

The compute path is the in-tree CUDA library only: if it is missing or no
CUDA device is usable the calls raise; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "PeriodSearch",
    "PeriodSearchBatch",
    "PeriodSearchError",
    "RECORD_DTYPE",
    "FIT_DTYPE",
    "load_library",
    "prepare",
    "precalc",
    "start",
    "unprepare",
    "format_record",
    "open_many",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libps_b200.so")
EXE_PATH = os.path.join(_HERE, "period_search_b200")

PS_OK, PS_ERR_IO, PS_ERR_LIMIT, PS_ERR_CUDA, PS_ERR_SINGULAR, PS_ERR_ARG, PS_ERR_DEVICE_LOOP = range(7)
PS_FORM_FP64 = 0
PS_FORM_MIXED = 1
PS_FORM_FAST = 2

RECORD_DTYPE = np.dtype(
    [("period_h", "f8"), ("rms", "f8"), ("chi2", "f8"), ("dark_pct", "f8"), ("lambda_deg", "f8"), ("beta_deg", "f8")]
)


class _FitResult(ctypes.Structure):
    _fields_ = [
        ("dev", ctypes.c_double),
        ("dark", ctypes.c_double),
        ("totarea", ctypes.c_double),
        ("period_d", ctypes.c_double),
        ("lambda_deg", ctypes.c_double),
        ("beta_deg", ctypes.c_double),
        ("chisq", ctypes.c_double),
        ("niter", ctypes.c_int),
        ("status", ctypes.c_int),
    ]


FIT_DTYPE = np.dtype([(n, "f8" if t is ctypes.c_double else "i4") for n, t in _FitResult._fields_])

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class _ProblemDesc(ctypes.Structure):
    _fields_ = [
        ("n_points", ctypes.c_int),
        ("n_lc", ctypes.c_int),
        ("lc_points", _I),
        ("lc_relative", _I),
        ("tim", _D),
        ("ee", _D),
        ("ee0", _D),
        ("brightness", _D),
        ("sig", _D),
        ("weight", _D),
        ("per_start", ctypes.c_double),
        ("per_step_coef", ctypes.c_double),
        ("per_end", ctypes.c_double),
        ("ia_prd", ctypes.c_int),
        ("phi0_rad", ctypes.c_double),
        ("conw", ctypes.c_double),
        ("lmax", ctypes.c_int),
        ("mmax", ctypes.c_int),
        ("nrows", ctypes.c_int),
        ("par", ctypes.c_double * 3),
        ("ia_par", ctypes.c_int * 3),
        ("cl", ctypes.c_double),
        ("ia_cl", ctypes.c_int),
        ("stop_condition", ctypes.c_double),
        ("n_iter_min", ctypes.c_int),
        ("alamda_incr", ctypes.c_double),
        ("alamda_start", ctypes.c_double),
        ("jd_min", ctypes.c_double),
        ("jd_max", ctypes.c_double),
        ("escl", ctypes.c_double),
    ]


class PeriodSearchError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"period_search_b200 error {code}: {msg}")
        self.code = code


_lib = None

# every symbol include/period_search_b200.h declares
EXPORTS = (
    "ps_open_file", "ps_open", "ps_close", "ps_precalc", "ps_set_conw_r", "ps_n_periods", "ps_scan",
    "ps_scan_device", "ps_fit", "ps_mrqcof", "ps_model", "ps_info", "ps_get_array", "ps_open_host_only",
    "ps_format_record", "ps_last_error", "ps_kernel_launches", "ps_scan_device_noalloc",
    "ps_batch_open", "ps_batch_scan", "ps_batch_scan_device", "ps_batch_fit_times", "ps_batch_close",
    "ps_fp64_tensor_peak", "ps_chi2_grad", "ps_gn_product", "ps_fit_jfree", "ps_set_tiles", "ps_autotune",
    "ps_release_cached_memory",
)


def load_library(path: str | None = None):
    """Load (once) the in-tree native library; raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise PeriodSearchError(PS_ERR_IO, f"native library not built: {p} (run python -m periodsearch_b200.build)")
    lib = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    sig = {
        "ps_open_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
        "ps_open": (ctypes.c_int, [ctypes.POINTER(_ProblemDesc), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
        "ps_open_host_only": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vp)]),
        "ps_close": (None, [vp]),
        "ps_precalc": (ctypes.c_int, [vp, _D]),
        "ps_set_conw_r": (ctypes.c_int, [vp, ctypes.c_double]),
        "ps_n_periods": (ctypes.c_int, [vp]),
        "ps_scan": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
        "ps_scan_device": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, vp]),
        "ps_scan_device_noalloc": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, vp]),
        "ps_fit": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_FitResult), _D]),
        "ps_mrqcof": (ctypes.c_int, [vp, _D, _D, _D, _D]),
        "ps_model": (ctypes.c_int, [vp, _D, _D, _D]),
        "ps_info": (ctypes.c_int, [vp, _I, _D]),
        "ps_get_array": (ctypes.c_int, [vp, ctypes.c_char_p, _D]),
        "ps_format_record": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]),
        "ps_last_error": (ctypes.c_char_p, []),
        "ps_batch_open": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]),
        "ps_batch_scan": (ctypes.c_int, [vp, _I, _I, vp]),
        "ps_batch_scan_device": (ctypes.c_int, [vp, _I, _I, vp, vp]),
        "ps_batch_fit_times": (ctypes.c_int, [vp, _D, _D]),
        "ps_batch_close": (None, [vp]),
        "ps_kernel_launches": (ctypes.c_longlong, []),
        "ps_fp64_tensor_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
        "ps_chi2_grad": (ctypes.c_int, [vp, _D, _D, _D]),
        "ps_set_tiles": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "ps_autotune": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _D]),
        "ps_gn_product": (ctypes.c_int, [vp, _D, _D, _D]),
        "ps_fit_jfree": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_FitResult), _D]),
        "ps_release_cached_memory": (None, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _check(rc):
    if rc != PS_OK:
        raise PeriodSearchError(rc, load_library().ps_last_error().decode())


def _dptr(a):
    return a.ctypes.data_as(_D)


class PeriodSearch:
    """One asteroid's scan on one GPU (the context of the C ABI)."""

    def __init__(self, path: str | None = None, *, device: int = 0, form: int = PS_FORM_FP64,
                 host_only: bool = False, desc: dict | None = None):
        lib = load_library()
        self._lib = lib
        self._h = ctypes.c_void_p()
        if desc is not None:
            self._keep, d = _make_desc(desc)
            _check(lib.ps_open(ctypes.byref(d), device, form, ctypes.byref(self._h)))
        elif host_only:
            _check(lib.ps_open_host_only(os.fsencode(path), ctypes.byref(self._h)))
        else:
            _check(lib.ps_open_file(os.fsencode(path), device, form, ctypes.byref(self._h)))
        ints = (ctypes.c_int * 8)()
        dbls = (ctypes.c_double * 8)()
        lib.ps_info(self._h, ints, dbls)
        (self.n_points, self.n_lc, self.numfac, self.ncoef, self.ma, self.mfit, self.n_periods) = list(ints)[:7]
        self.ncb = (self.ncoef + 7) // 8 * 8  # shape columns padded to 8 on the device
        self.escl, self.conw_r, self.freq_start, self.freq_end, self.freq_step = list(dbls)[:5]

    # -- lifetime
    def close(self):
        if self._h:
            self._lib.ps_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the scan (CUDAPrecalc / CUDAStart)
    def precalc(self) -> float:
        v = ctypes.c_double()
        _check(self._lib.ps_precalc(self._h, ctypes.byref(v)))
        self.conw_r = v.value
        ints = (ctypes.c_int * 8)()
        self._lib.ps_info(self._h, ints, None)
        self.prepass_fits = ints[7]
        return v.value

    def set_conw_r(self, conw_r: float):
        _check(self._lib.ps_set_conw_r(self._h, float(conw_r)))
        self.conw_r = float(conw_r)

    def scan(self, n_from: int = 1, n_to: int | None = None) -> np.ndarray:
        n_to = self.n_periods if n_to is None else n_to
        out = np.zeros(max(n_to - n_from + 1, 0), dtype=RECORD_DTYPE)
        _check(self._lib.ps_scan(self._h, n_from, n_to, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def scan_device(self, n_from: int, n_to: int, d_out_ptr: int, stream_ptr: int = 0):
        _check(self._lib.ps_scan_device(self._h, n_from, n_to, ctypes.c_void_p(d_out_ptr),
                                        ctypes.c_void_p(stream_ptr or None)))

    def fit(self, freq: float, pole: int, params: bool = False):
        """One LM fit (ps_fit); with params=True also its final parameters."""
        return self._fit(self._lib.ps_fit, freq, pole, params)

    def fit_jfree(self, freq: float, pole: int, params: bool = False):
        """The same fit Jacobian-free (ps_fit_jfree: matrix-free kernels)."""
        return self._fit(self._lib.ps_fit_jfree, freq, pole, params)

    def _fit(self, fn, freq, pole, params):
        r = _FitResult()
        cg = np.zeros(self.ma)
        _check(fn(self._h, float(freq), int(pole), ctypes.byref(r), _dptr(cg) if params else None))
        rec = np.array([tuple(getattr(r, n) for n, _ in _FitResult._fields_)], dtype=FIT_DTYPE)[0]
        return (rec, cg) if params else rec

    def mrqcof(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        alpha = np.zeros((self.mfit, self.mfit))
        beta = np.zeros(self.mfit)
        chi = np.zeros(1)
        _check(self._lib.ps_mrqcof(self._h, _dptr(a), _dptr(alpha), _dptr(beta), _dptr(chi)))
        return alpha, beta, float(chi[0])

    def model(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        y = np.zeros(self.n_points + 3)
        J = np.zeros((self.n_points + 3, self.ma))
        _check(self._lib.ps_model(self._h, _dptr(a), _dptr(y), _dptr(J)))
        return y, J

    def set_tiles(self, fch: int, rt: int, sortseg: int):
        """Tile shapes (results unchanged): facets per staged chunk and alpha
        rows per tile of the fast form, points sorted together."""
        _check(self._lib.ps_set_tiles(self._h, fch, rt, sortseg))

    def autotune(self, n_periods: int = 30):
        """Time candidate tile shapes on periods 1..n_periods, keep the
        fastest; returns ((fch, rt, sortseg), seconds)."""
        t = (ctypes.c_int * 3)()
        sec = ctypes.c_double()
        _check(self._lib.ps_autotune(self._h, n_periods, t, ctypes.byref(sec)))
        return (t[0], t[1], t[2]), sec.value

    def chi2_grad(self, a):
        """Matrix-free (chi2, beta) at a; the chi2 gradient over the free
        parameters is -2 beta."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        beta = np.zeros(self.mfit)
        x2 = np.zeros(1)
        _check(self._lib.ps_chi2_grad(self._h, _dptr(a), _dptr(x2), _dptr(beta)))
        return float(x2[0]), beta

    def gn_product(self, a, v):
        """Matrix-free J^T W (J v) at a for v over the free parameters."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros(self.mfit)
        _check(self._lib.ps_gn_product(self._h, _dptr(a), _dptr(v), _dptr(out)))
        return out

    def array(self, name: str) -> np.ndarray:
        size = {"nor": 3 * self.numfac, "darea": self.numfac, "dsph": self.numfac * self.ncoef,
                "cg_first": self.ncoef, "ia": self.ma, "tim": self.n_points, "ee": 3 * self.n_points,
                "ee0": 3 * self.n_points, "brightness": self.n_points + 3, "sig": self.n_points + 3,
                "weight": self.n_points + 3, "at": self.numfac, "af": self.numfac, "ifp": 3 * self.numfac}[name]
        out = np.zeros(size)
        n = self._lib.ps_get_array(self._h, name.encode(), _dptr(out))
        if n < 0:
            raise PeriodSearchError(PS_ERR_ARG, "unknown array " + name)
        return out[:n]


class PeriodSearchBatch:
    """Several asteroids (PeriodSearch contexts with the same lmax, mmax,
    nrows, device and FP64 form) scanned in one persistent launch."""

    def __init__(self, contexts):
        self._lib = load_library()
        self._ctx = list(contexts)
        arr = (ctypes.c_void_p * len(self._ctx))(*[c._h.value for c in self._ctx])
        self._h = ctypes.c_void_p()
        _check(self._lib.ps_batch_open(arr, len(self._ctx), ctypes.byref(self._h)))

    def _ranges(self, n_from, n_to):
        a = np.ascontiguousarray(n_from, dtype=np.int32)
        b = np.ascontiguousarray(n_to, dtype=np.int32)
        if a.shape != (len(self._ctx),) or b.shape != a.shape:
            raise PeriodSearchError(PS_ERR_ARG, "one period range per asteroid")
        return a, b

    def scan(self, n_from, n_to):
        """Records per asteroid (list of arrays)."""
        a, b = self._ranges(n_from, n_to)
        counts = (b - a + 1).astype(np.int64)
        out = np.zeros(int(counts.sum()), dtype=RECORD_DTYPE)
        _check(self._lib.ps_batch_scan(self._h, a.ctypes.data_as(_I), b.ctypes.data_as(_I),
                                       out.ctypes.data_as(ctypes.c_void_p)))
        return np.split(out, np.cumsum(counts)[:-1])

    def scan_device(self, n_from, n_to, d_out_ptr: int, stream_ptr: int = 0):
        a, b = self._ranges(n_from, n_to)
        _check(self._lib.ps_batch_scan_device(self._h, a.ctypes.data_as(_I), b.ctypes.data_as(_I),
                                              ctypes.c_void_p(d_out_ptr), ctypes.c_void_p(stream_ptr or None)))

    def fit_times(self):
        """(busy_ms, done_ms) per asteroid of the last scan: summed fit time,
        and wall time from the scan's first fit start to the asteroid's last
        fit end."""
        busy = np.zeros(len(self._ctx))
        done = np.zeros(len(self._ctx))
        _check(self._lib.ps_batch_fit_times(self._h, _dptr(busy), _dptr(done)))
        return busy, done

    @staticmethod
    def autotune(contexts, n_from, n_to, n_periods: int = 60):
        """Tile shapes for a batch: tune one asteroid (the work-weighted median
        by points x periods) with ps_autotune, then time one batch scan of
        [n_from, n_to] with those tiles and with the defaults and keep the
        faster -- one asteroid's optimum need not hold for a whole persistent
        batch.  Sets the tiles on every context; returns (tiles, seconds)."""
        import time

        ctxs = list(contexts)
        nf = np.asarray(n_from)
        nt = np.asarray(n_to)
        work = np.array([c.n_points for c in ctxs], dtype=np.float64) * (nt - nf + 1)
        order = np.argsort(work)
        k = int(order[np.searchsorted(np.cumsum(work[order]), 0.5 * work.sum())])
        tuned, _ = ctxs[k].autotune(n_periods)
        best, tbest = None, None
        for tiles in dict.fromkeys([(40, 32, 1024), tuple(tuned)]):
            for c in ctxs:
                c.set_tiles(*tiles)
            b = PeriodSearchBatch(ctxs)
            try:
                b.scan(nf, nt)  # graph capture and warm-up
                t0 = time.perf_counter()
                b.scan(nf, nt)
                dt = time.perf_counter() - t0
            finally:
                b.close()
            if tbest is None or dt < tbest:
                best, tbest = tiles, dt
        for c in ctxs:
            c.set_tiles(*best)
        return best, tbest

    def close(self):
        if self._h:
            self._lib.ps_batch_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _make_desc(d: dict):
    keep = {}

    def arr(name, dtype):
        a = np.ascontiguousarray(d[name], dtype=dtype)
        keep[name] = a
        return a.ctypes.data_as(_D if dtype == np.float64 else _I)

    s = _ProblemDesc()
    s.n_points = int(len(d["tim"]))
    s.n_lc = int(len(d["lc_points"]))
    s.lc_points = arr("lc_points", np.int32)
    s.lc_relative = arr("lc_relative", np.int32)
    for k in ("tim", "ee", "ee0", "brightness", "sig", "weight"):
        setattr(s, k, arr(k, np.float64))
    for k in ("per_start", "per_step_coef", "per_end", "phi0_rad", "conw", "cl", "stop_condition",
              "alamda_incr", "alamda_start", "jd_min", "jd_max", "escl"):
        setattr(s, k, float(d[k]))
    for k in ("ia_prd", "lmax", "mmax", "nrows", "ia_cl", "n_iter_min"):
        setattr(s, k, int(d[k]))
    s.par = (ctypes.c_double * 3)(*d["par"])
    s.ia_par = (ctypes.c_int * 3)(*d["ia_par"])
    keep["_struct"] = s
    return keep, s


def open_many(paths, *, device: int = 0, form: int = PS_FORM_FP64, conw_r=None, threads: int | None = None):
    """Open one context per input file concurrently (for a batch): each
    asteroid's host setup -- parsing, the ellipsoid fit, the facet and
    spherical-harmonic tables (period_search_BOINC.cpp:277-485, sphfunc.c,
    ellfit.c) -- and its uploads run on a pool of host threads (the C calls
    release the GIL; facet-grid tables shared by asteroids with the same
    nrows/lmax/mmax are built once).  conw_r: None leaves it unset, "start"
    uses each asteroid's pre-pass start value conw/escl^2, a number sets it.
    Returns the contexts in the order of `paths`."""
    from concurrent.futures import ThreadPoolExecutor

    paths = list(paths)

    def one(p):
        c = PeriodSearch(p, device=device, form=form)
        if conw_r == "start":
            c.set_conw_r(c.conw_r)
        elif conw_r is not None:
            c.set_conw_r(float(conw_r))
        return c

    n = threads or min(len(paths), os.cpu_count() or 1, 32)
    if n <= 1:
        return [one(p) for p in paths]
    with ThreadPoolExecutor(n) as ex:
        return list(ex.map(one, paths))


def fp64_tensor_peak(device: int = 0) -> float:
    """Measured FP64 tensor-core throughput of the device, TFLOP/s."""
    v = ctypes.c_double()
    _check(load_library().ps_fp64_tensor_peak(device, ctypes.byref(v)))
    return v.value


def format_record(rec, first_line: bool = False, conw_line: float = 0.0) -> str:
    """One output line in the reference format (period_search_BOINC.cpp:926-931)."""
    lib = load_library()
    arr = np.array([tuple(rec)], dtype=RECORD_DTYPE)
    buf = ctypes.create_string_buffer(256)
    lib.ps_format_record(arr.ctypes.data_as(ctypes.c_void_p), int(first_line), float(conw_line), buf, 256)
    return buf.value.decode()


# -- module-level mirror of the reference's process-global operator API
_default: PeriodSearch | None = None


def prepare(path: str, device: int = 0) -> int:
    """CUDAPrepare: parse period_search_in and upload it.  Returns 1 on
    success like the reference (start_CUDA.cu:232-237), raises otherwise."""
    global _default
    if _default is not None:
        _default.close()
    _default = PeriodSearch(path, device=device)
    return 1


def precalc() -> float:
    """CUDAPrecalc: the convexity-weight pre-pass; returns conw_r."""
    if _default is None:
        raise PeriodSearchError(PS_ERR_ARG, "prepare() first")
    return _default.precalc()


def start(n_start_from: int = 1, n_to: int | None = None) -> np.ndarray:
    """CUDAStart: scan from trial period n_start_from; returns the records."""
    if _default is None:
        raise PeriodSearchError(PS_ERR_ARG, "prepare() first")
    return _default.scan(n_start_from, n_to)


def unprepare() -> None:
    """CUDAUnprepare: release the device state."""
    global _default
    if _default is not None:
        _default.close()
        _default = None
