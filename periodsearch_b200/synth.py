"""Seeded synthetic ``period_search_in`` generator.

The reference publishes no benchmark inputs, so every workload here is a
seeded synthetic asteroid written in the reference's own input format
(period_search/period_search_BOINC.cpp:277-427):

* shape: triaxial ellipsoid with axes 1 : U(0.6,0.9) : U(0.4,0.7), its
  Gaussian-image area density multiplied by exp(sum of orthonormal real
  spherical harmonics up to the true lmax, coefficients N(0, 0.1^2));
* spin: pole lambda U(0,360) deg, beta U(-90,90) deg, period U(4,12) h;
* geometry: Sun and Earth vectors from circular orbits (asteroid at 2.5 AU,
  inclined 8 deg to the ecliptic so that the (lambda, beta) / (lambda, -beta)
  mirror pair is not exactly degenerate; Earth at 1 AU), epochs at solar
  elongation > 60 deg; the phase angle stays below asin(1/2.5) = 23.6 deg;
* brightness: Lambert (c_L = 0.1) + Lommel-Seeliger (c_LS = 1) on a fine
  facet grid (4000 normals), phase function 1 + a exp(-alpha/d) + k alpha
  with a=0.5, d=0.1, k=-0.5, multiplicative Gaussian noise;
* dense lightcurves: one night each (points over 8 h), flag 0 (relative);
  sparse sets: uniform over the baseline, flag 1 (calibrated).

The rotation convention is the reference's (blmatrix.c / matrix.c): body
coordinates = R_z(phi) . R_(beta',lambda) . ecliptic, phi = omega t + phi0,
beta' = 90 deg - beta, omega = 2 pi 24 / P[h] rad/day.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

__all__ = ["Workload", "make_workload", "write_input", "CONFIGS", "n_periods_of"]


@dataclasses.dataclass
class Workload:
    name: str
    text: str  # the period_search_in file contents
    n_points: int
    n_lc: int
    lmax: int
    nrows: int
    n_periods: int
    true_period_h: float
    true_pole: tuple


def _real_sph_basis(lmax, theta, phi):
    from scipy.special import sph_harm_y

    cols = []
    for l in range(1, lmax + 1):
        for m in range(-l, l + 1):
            y = sph_harm_y(l, abs(m), theta, phi)
            if m > 0:
                cols.append(math.sqrt(2.0) * (-1) ** m * y.real)
            elif m < 0:
                cols.append(math.sqrt(2.0) * (-1) ** m * y.imag)
            else:
                cols.append(y.real)
    return np.stack(cols, axis=1) if cols else np.zeros((theta.size, 0))


def _fib_sphere(k):
    i = np.arange(k) + 0.5
    z = 1.0 - 2.0 * i / k
    r = np.sqrt(1.0 - z * z)
    ph = math.pi * (1.0 + 5.0**0.5) * i
    n = np.stack([r * np.cos(ph), r * np.sin(ph), z], axis=1)
    return n


def _rot_pole(beta_p, lam):
    cb, sb, cl, sl = math.cos(beta_p), math.sin(beta_p), math.cos(lam), math.sin(lam)
    return np.array([[cb * cl, cb * sl, -sb], [-sl, cl, 0.0], [sb * cl, sb * sl, cb]])


def _orbit_pos(radius, period_days, incl, node, phase0, t):
    ang = phase0 + 2 * math.pi * t / period_days
    x = radius * np.cos(ang)
    y = radius * np.sin(ang)
    # rotate by inclination about the x axis then by the node about z
    y2, z2 = y * math.cos(incl), y * math.sin(incl)
    xc, yc = x * math.cos(node) - y2 * math.sin(node), x * math.sin(node) + y2 * math.cos(node)
    return np.stack([xc, yc, z2], axis=-1)


def n_periods_of(p_start, step_coef, p_end, jd_min, jd_max):
    """Trial-period count exactly as period_search_BOINC.cpp:784-786,807."""
    f_start = 1 / p_start
    f_end = 1 / p_end
    f_step = 0.5 / (jd_max - jd_min) / 24 * step_coef
    return int((f_start - f_end) / f_step) + 1


class _Body:
    def __init__(self, rng, true_lmax, phase=(0.5, 0.1, -0.5), c_l=0.1):
        self.axes = np.array([1.0, rng.uniform(0.6, 0.9), rng.uniform(0.4, 0.7)])
        self.normals = _fib_sphere(4000)
        th = np.arccos(np.clip(self.normals[:, 2], -1, 1))
        ph = np.arctan2(self.normals[:, 1], self.normals[:, 0])
        a, b, c = self.axes
        n = self.normals
        dens = (a * b * c) ** 2 / (a * a * n[:, 0] ** 2 + b * b * n[:, 1] ** 2 + c * c * n[:, 2] ** 2) ** 2
        basis = _real_sph_basis(true_lmax, th, ph)
        coef = rng.normal(0.0, 0.1, basis.shape[1])
        self.area = dens * np.exp(basis @ coef) * (4 * math.pi / n.shape[0])
        self.lam = math.radians(rng.uniform(0, 360))
        self.beta = math.radians(rng.uniform(-90, 90))
        self.period_h = rng.uniform(4, 12)
        self.phi0 = 0.0
        self.phase = phase
        self.c_l = c_l

    def brightness(self, t_rel, e_sun, e_earth):
        """Model brightness (unit distances) at times t_rel [day] for
        asteroid->Sun / asteroid->Earth unit vectors (ecliptic)."""
        omega = 24 * 2 * math.pi / self.period_h
        R0 = _rot_pole(math.pi / 2 - self.beta, self.lam)
        f = np.fmod(omega * t_rel + self.phi0, 2 * math.pi)
        cf, sf = np.cos(f), np.sin(f)
        # body frame: R_z(f) R0 v, for all epochs at once
        e0 = e_earth @ R0.T
        s0 = e_sun @ R0.T
        rot = lambda v: np.stack([cf * v[:, 0] + sf * v[:, 1], -sf * v[:, 0] + cf * v[:, 1], v[:, 2]], axis=1)
        e, es = rot(e0), rot(s0)
        out = np.empty(t_rel.shape[0])
        a, d, k = self.phase
        for i0 in range(0, t_rel.shape[0], 512):
            sl = slice(i0, i0 + 512)
            mu = e[sl] @ self.normals.T
            mu0 = es[sl] @ self.normals.T
            vis = (mu > 1e-8) & (mu0 > 1e-8)
            s = np.where(vis, mu * mu0 * (self.c_l + 1.0 / np.where(vis, mu + mu0, 1.0)), 0.0)
            alpha = np.arccos(np.clip(np.sum(e_earth[sl] * e_sun[sl], 1), -1, 1))
            out[sl] = (1 + a * np.exp(-alpha / d) + k * alpha) * (s @ self.area)
        return out


def _observable_epochs(rng, n, t0, span, ast, earth_fn, min_elong=60.0):
    out = []
    while len(out) < n:
        t = t0 + rng.uniform(0, span, size=4 * n)
        a = ast(t)
        e = earth_fn(t)
        to_ast = a - e
        to_sun = -e
        cosel = np.sum(to_ast * to_sun, 1) / np.linalg.norm(to_ast, axis=1) / np.linalg.norm(to_sun, axis=1)
        ok = np.degrees(np.arccos(np.clip(cosel, -1, 1))) > min_elong
        out.extend(t[ok].tolist())
    return np.sort(np.array(out[:n]))


def make_workload(
    name: str,
    seed: int,
    *,
    dense_lcs: int,
    dense_pts: int,
    sparse_sets: int = 1,
    sparse_pts: int,
    years: float,
    true_lmax: int,
    fit_lmax: int,
    nrows: int,
    noise: float,
    n_periods: int | None = None,
    period_range_h: tuple | None = None,
    step_coef: float = 0.5,
    stop_condition: float = 50,
    n_iter_min: int = 10,
    conw: float = 0.1,
) -> Workload:
    """Build one synthetic asteroid and its period_search_in text.

    Either ``n_periods`` (a window of exactly that many trial periods
    centred on the true period, step_coef as given) or ``period_range_h``
    (a fixed range, the count following the reference's step rule)."""
    rng = np.random.default_rng(seed)
    body = _Body(rng, true_lmax)
    jd_start = 2451545.0 + float(rng.uniform(0, 1000))
    span = years * 365.25
    incl, node, ph_a, ph_e = math.radians(8.0), rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi)
    ast = lambda t: _orbit_pos(2.5, 365.25 * 2.5**1.5, incl, node, ph_a, t - 2451545.0)
    earth = lambda t: _orbit_pos(1.0, 365.25, 0.0, 0.0, ph_e, t - 2451545.0)

    lcs = []  # (flag, times)
    nights = _observable_epochs(rng, dense_lcs, jd_start, span - 1.0, ast, earth)
    for t0 in nights:
        lcs.append((0, np.sort(t0 + rng.uniform(0, 8.0 / 24, size=dense_pts))))
    for _ in range(sparse_sets):
        if sparse_pts > 0:
            lcs.append((1, _observable_epochs(rng, sparse_pts, jd_start, span, ast, earth)))

    rows = []
    for flag, t in lcs:
        pa, pe = ast(t), earth(t)
        e_sun = -pa  # asteroid -> Sun
        e_earth = pe - pa  # asteroid -> Earth
        un = lambda v: v / np.linalg.norm(v, axis=1, keepdims=True)
        br = body.brightness(t - jd_start, un(e_sun), un(e_earth))
        br = br * (1.0 + noise * rng.standard_normal(br.shape[0]))
        rows.append((flag, t, br, e_sun, e_earth))

    all_t = np.concatenate([r[1] for r in rows])
    jd_min, jd_max = float(all_t.min()), float(all_t.max())
    # the file stores JD with 6 decimals; use the parsed values for the grid
    jd_min = float("%.6f" % jd_min)
    jd_max = float("%.6f" % jd_max)
    if n_periods is not None:
        f_step = 0.5 / (jd_max - jd_min) / 24 * step_coef
        f_true = 1.0 / body.period_h
        half = (n_periods - 1) / 2.0 + 0.2
        p_start = float("%.10f" % (1.0 / (f_true + half * f_step)))
        p_end = float("%.10f" % (1.0 / (f_true - half * f_step)))
        got = n_periods_of(p_start, step_coef, p_end, jd_min, jd_max)
        # nudge the end of the window until the count is exact
        for _ in range(100):
            if got == n_periods:
                break
            p_end = float("%.10f" % (p_end * (1 + (1e-7 if got < n_periods else -1e-7))))
            got = n_periods_of(p_start, step_coef, p_end, jd_min, jd_max)
        assert got == n_periods, (got, n_periods)
    else:
        p_start, p_end = period_range_h
        got = n_periods_of(p_start, step_coef, p_end, jd_min, jd_max)

    lines = [
        "%.10f %g %.10f 1\tperiod_start period_step period_end fixed/free" % (p_start, step_coef, p_end),
        "0.0\t\t\t\tinitial epoch",
        "0.0\t\t\t\tinitial rotation angle",
        "%g\t\t\t\tconvexity weight" % conw,
        "%d %d\t\t\t\tdegree and order of spherical harmonics" % (fit_lmax, fit_lmax),
        "%d\t\t\t\tnumber of rows" % nrows,
        "0.5\t1\t\t\tscattering parameters",
        "0.1\t1",
        "-0.5\t1",
        "0.1\t0\t\t\tLS coeff",
        "%g\t\t\t\titeration stop condition" % stop_condition,
        "%d\t\t\t\tminimum number of iterations (only if the above value < 1)" % n_iter_min,
        "5\t\t\t\tAlamda multiplicative factor",
        "0.1\t\t\t\tAlamda initial value",
        "%d" % len(rows),
    ]
    npts = 0
    for flag, t, br, es, ee in rows:
        lines.append("%d %d synthetic %s" % (t.shape[0], flag, "sparse" if flag else "dense"))
        for i in range(t.shape[0]):
            lines.append(
                "%.6f %.6e %.6e %.6e %.6e %.6e %.6e %.6e"
                % (t[i], br[i], es[i, 0], es[i, 1], es[i, 2], ee[i, 0], ee[i, 1], ee[i, 2])
            )
        npts += t.shape[0]
    text = "\n".join(lines) + "\n"
    return Workload(
        name=name,
        text=text,
        n_points=npts,
        n_lc=len(rows),
        lmax=fit_lmax,
        nrows=nrows,
        n_periods=got,
        true_period_h=body.period_h,
        true_pole=(math.degrees(body.lam), math.degrees(body.beta)),
    )


def _c1(seed=1, n_periods=200):
    return make_workload("c1_lmax3_n500_f288", seed, dense_lcs=6, dense_pts=50, sparse_pts=200, years=8,
                         true_lmax=3, fit_lmax=3, nrows=6, noise=0.02, n_periods=n_periods)


def _c2(seed=2, n_periods=None, step_coef=2.15):
    kw = dict(n_periods=n_periods) if n_periods else dict(period_range_h=(2.0, 100.0))
    return make_workload("c2_lmax6_n760_f800", seed, dense_lcs=2, dense_pts=80, sparse_pts=600, years=10,
                         true_lmax=6, fit_lmax=6, nrows=10, noise=0.03, step_coef=step_coef, **kw)


def _tiny(seed=7, n_periods=4):
    return make_workload("tiny_lmax2_n60_f72", seed, dense_lcs=2, dense_pts=20, sparse_pts=20, years=4,
                         true_lmax=2, fit_lmax=2, nrows=3, noise=0.02, n_periods=n_periods)


def _tiny_rel(seed=8, n_periods=3):
    """All-relative variant (exercises ia[1] = 0, mrqcof normalisation)."""
    return make_workload("tinyrel_lmax2_n60_f72", seed, dense_lcs=3, dense_pts=20, sparse_pts=0, years=3,
                         true_lmax=2, fit_lmax=2, nrows=3, noise=0.02, n_periods=n_periods)


def c4_asteroid(i: int, periods: int | None = None):
    """Asteroid i of the uneven multi-asteroid batch: N log-uniform in
    100-5000, dense/sparse split U(0,1) (dense nights of 40-80 points),
    lmax = mmax = 6, nrows = 10, a period window of U(5 %, 50 %) of 2-100 h
    around the true period at the reference step rule, and the per-fit
    convergence stop rule (stop_condition 1e-4 on the rms improvement,
    n_iter_min 5, capped at 100 iterations by the reference)."""
    rng = np.random.default_rng(40000 + i)
    n = int(round(math.exp(rng.uniform(math.log(100), math.log(5000)))))
    dense_frac = rng.uniform(0, 1)
    per_night = int(rng.integers(40, 81))
    n_dense = int(round(n * dense_frac / per_night))
    sparse = max(n - n_dense * per_night, 0)
    if n_dense == 0 and sparse == 0:
        sparse = n
    width = rng.uniform(0.05, 0.5) * 98.0
    w = make_workload(f"c4_{i}", 40000 + i, dense_lcs=n_dense, dense_pts=per_night, sparse_pts=sparse, years=8,
                      true_lmax=6, fit_lmax=6, nrows=10, noise=0.03, n_periods=periods or 16,
                      stop_condition=1e-4, n_iter_min=5)
    # the full window: P_true +- width/2 clipped to 2-100 h (the count follows
    # the step rule); tests and the bench scan a slice of it
    return w, width


CONFIGS = {"tiny": _tiny, "tiny_rel": _tiny_rel, "c1": _c1, "c2": _c2}


def write_input(w: Workload, directory: str) -> str:
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "period_search_in")
    with open(path, "w") as f:
        f.write(w.text)
    return path
