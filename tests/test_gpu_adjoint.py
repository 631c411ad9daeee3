"""Matrix-free derivatives (ps_chi2_grad, ps_gn_product) through the C ABI.

* against the explicit Jacobian of the same library (ps_mrqcof: chi2, beta,
  alpha), which is itself held to the oracle at 1e-11: chi2, beta and
  J^T W (J v) = alpha v agree to 1e-10 (normwise; fused arithmetic in a
  different order);
* against central finite differences of chi2 (from ps_mrqcof) with a
  relative step of 1e-6 (1e-10 for the rotation rate: over a multi-year
  baseline the visibility-mask kinks of chi2(omega) are so dense that the
  reference's own chi2 only converges to its analytic derivative below a
  1e-10 step -- on c1, -169.9 / -153.9 / -156.9 / -161.5322 at 1e-7 / 1e-8 /
  1e-9 / 1e-10 against -161.5324): the gradient -2 beta agrees to 1e-4 per
  component;
* wrapped in a torch.autograd.Function (test harness only): autograd's
  gradient of chi2 is the matrix-free one, and its double-backward-free
  Gauss-Newton product matches alpha v;
* at the matrix-free configuration's full size (N = 20 000, 2048 facets,
  81 coefficients), where one Gauss-Newton product is timed against one
  explicit evaluation.
"""
import time

import numpy as np
import pytest

from conftest import golden_path
from periodsearch_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _open(native, oracle_lib, path):
    o = oracle_lib.Oracle(path)
    o.set_conw_r(o.conw_r)
    g = native.PeriodSearch(path, form=native.PS_FORM_FAST)
    g.set_conw_r(o.conw_r)
    return g, o


def _points(o, rng):
    ia = np.array(o.array("ia")) > 0
    out = []
    for n, pole in ((1, 1), (o.n_periods, 7)):
        a = o.initial_parameters(o.freq(n), pole)
        out.append(a)
        out.append(a + rng.normal(0, 1e-3, a.shape) * (np.abs(a) + 0.1) * ia)
    return out, np.nonzero(ia)[0]


@pytest.mark.parametrize("name", ["tiny", "tiny_rel", "c1"])
def test_matches_explicit_jacobian(native, oracle_lib, name):
    g, o = _open(native, oracle_lib, golden_path(name))
    rng = np.random.default_rng(11)
    pts, free = _points(o, rng)
    for a in pts:
        alpha, beta, x2 = g.mrqcof(a)
        x2m, betam = g.chi2_grad(a)
        assert abs(x2m - x2) <= TOL * abs(x2), (name, x2m, x2)
        assert _rel(betam, beta) <= TOL, (name, _rel(betam, beta))
        for _ in range(3):
            v = rng.normal(size=len(free))
            assert _rel(g.gn_product(a, v), alpha @ v) <= TOL, name
    g.close()


def _fd_grad(g, a, free):
    grad = np.zeros(len(free))
    C = g.ncoef
    for i, k in enumerate(free):
        h = (1e-10 if k == C + 2 else 1e-6) * max(abs(a[k]), 0.1)
        ap, am = a.copy(), a.copy()
        ap[k] += h
        am[k] -= h
        grad[i] = (g.mrqcof(ap)[2] - g.mrqcof(am)[2]) / (2 * h)
    return grad


@pytest.mark.parametrize("name", ["tiny", "tiny_rel", "c1"])
def test_gradient_vs_finite_differences(native, oracle_lib, name):
    g, o = _open(native, oracle_lib, golden_path(name))
    pts, free = _points(o, np.random.default_rng(3))
    for a in pts[:2]:
        _, beta = g.chi2_grad(a)
        grad = -2 * beta
        fd = _fd_grad(g, a, free)
        err = np.abs(fd - grad)
        assert np.all(err <= 1e-4 * np.abs(grad) + 1e-7 * np.linalg.norm(grad)), (name, np.max(err / (np.abs(grad) + 1e-300)))
    g.close()


def test_autograd_function(native, oracle_lib):
    torch = pytest.importorskip("torch")
    g, o = _open(native, oracle_lib, golden_path("c1"))
    pts, free = _points(o, np.random.default_rng(9))
    base = pts[1]

    class Chi2(torch.autograd.Function):
        """chi2 of the free parameters; backward through the adjoint kernel."""

        @staticmethod
        def forward(ctx, x):
            a = base.copy()
            a[free] = x.detach().cpu().numpy()
            x2, beta = g.chi2_grad(a)
            ctx.save_for_backward(torch.from_numpy(-2 * beta))
            ctx.a = a
            return torch.tensor(x2, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad

    x = torch.tensor(base[free], dtype=torch.float64, requires_grad=True)
    y = Chi2.apply(x)
    (gx,) = torch.autograd.grad(y, x)
    alpha, beta, x2 = g.mrqcof(base)
    assert abs(y.item() - x2) <= TOL * x2
    assert _rel(gx.numpy(), -2 * beta) <= TOL
    fd = _fd_grad(g, base, free)
    assert np.all(np.abs(fd - gx.numpy()) <= 1e-4 * np.abs(gx.numpy()) + 1e-7 * np.linalg.norm(gx.numpy()))
    # Gauss-Newton product as a vector-Jacobian-style operator
    v = torch.randn(len(free), dtype=torch.float64)
    assert _rel(g.gn_product(base, v.numpy()), alpha @ v.numpy()) <= TOL
    g.close()


def test_full_size_matrix_free(native, oracle_lib, tmp_path):
    w = synth.make_workload("large_full", 5, dense_lcs=40, dense_pts=100, sparse_pts=16000, years=10,
                            true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2)
    path = synth.write_input(w, str(tmp_path))
    g, o = _open(native, oracle_lib, path)
    assert (g.n_points, g.ncoef, g.mfit) == (20000, 81, 87)
    a = o.initial_parameters(o.freq(1), 2)
    alpha, beta, x2 = g.mrqcof(a)
    x2m, betam = g.chi2_grad(a)
    assert abs(x2m - x2) <= TOL * x2 and _rel(betam, beta) <= TOL
    v = np.random.default_rng(1).normal(size=g.mfit)
    assert _rel(g.gn_product(a, v), alpha @ v) <= TOL
    # one explicit evaluation (J and alpha) vs one matrix-free product
    t0 = time.perf_counter()
    for _ in range(3):
        g.mrqcof(a)
    t_explicit = (time.perf_counter() - t0) / 3
    t0 = time.perf_counter()
    for _ in range(3):
        g.gn_product(a, v)
    t_product = (time.perf_counter() - t0) / 3
    print(f"N=20000 F=2048 C=81: explicit evaluation {1e3 * t_explicit:.1f} ms (one CTA), "
          f"matrix-free product {1e3 * t_product:.1f} ms (whole GPU)")
    g.close()
