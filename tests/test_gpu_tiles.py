"""Tile shapes and the autotuner (ps_set_tiles, ps_autotune): every tile
choice leaves every result bit-identical -- the sums keep their order, only
the staging granularity and the point-to-warp assignment change."""
import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def _scan(g, n):
    return g.scan(1, n)


@pytest.mark.parametrize("name", ["tiny", "c1"])
def test_tiles_leave_results_unchanged(native, oracle_lib, name):
    o = oracle_lib.Oracle(golden_path(name))
    g = native.PeriodSearch(golden_path(name), form=native.PS_FORM_FAST)
    g.set_conw_r(o.conw_r)
    n = min(g.n_periods, 6)
    ref = _scan(g, n)
    for tiles in ((16, 16, 256), (64, 64, 1024), (4, 4, 32), (128, 8, 4096)):
        g.set_tiles(*tiles)
        got = _scan(g, n)
        assert np.array_equal(got.view(np.float64), ref.view(np.float64)), (name, tiles)
    best, sec = g.autotune(n)
    assert best[0] in (16, 32, 40, 48, 56, 64) and best[1] in (16, 32, 64) and best[2] in (256, 1024) and sec > 0
    assert np.array_equal(_scan(g, n).view(np.float64), ref.view(np.float64))
    g.close()


def test_sort_segment_in_reference_order_form(native, oracle_lib):
    o = oracle_lib.Oracle(golden_path("c1"))
    g = native.PeriodSearch(golden_path("c1"), form=native.PS_FORM_FP64)
    g.set_conw_r(o.conw_r)
    ref = _scan(g, 4)
    g.set_tiles(32, 32, 64)
    assert np.array_equal(_scan(g, 4).view(np.float64), ref.view(np.float64))
    g.close()


def test_bad_tiles_rejected(native):
    g = native.PeriodSearch(golden_path("tiny"), form=native.PS_FORM_FAST)
    for bad in ((3, 32, 1024), (32, 300, 1024), (32, 32, 1000), (256, 32, 1024)):
        with pytest.raises(native.PeriodSearchError):
            g.set_tiles(*bad)
    g.close()
