"""ps_scan_device_noalloc: the period scan for callers that cannot allocate
device memory while they run (a fixed pre-sized memory budget, a plugin
inside someone else's process, a service that cannot take cudaFree's
device-wide wait on its scan path).  It must
give the same records as ps_scan_device, call after call, with all of its
scratch in the library's fixed 64 MiB device array, and refuse a request that
does not fit there.  This file is collected last on purpose."""
import ctypes
import os
import shutil

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def _records(torch, ps, fn, g, n_from, n_to, stream=None):
    n = n_to - n_from + 1
    d = torch.full((n * 6,), float("nan"), dtype=torch.float64, device="cuda")
    rc = fn(g._h, n_from, n_to, ctypes.c_void_p(d.data_ptr()), stream)
    assert rc == ps.PS_OK, ps.load_library().ps_last_error()
    torch.cuda.synchronize()
    return d.view(n, 6).cpu().numpy()


def test_noalloc_scan_matches_scan_device(native):
    torch = pytest.importorskip("torch")
    ps = native
    lib = ps.load_library()
    g = ps.PeriodSearch(golden_path("c1"))
    g.set_conw_r(g.conw_r * 8)
    ref = _records(torch, ps, lib.ps_scan_device, g, 11, 40)
    first = _records(torch, ps, lib.ps_scan_device_noalloc, g, 11, 40)
    second = _records(torch, ps, lib.ps_scan_device_noalloc, g, 11, 40)
    for got in (first, second):
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
    # a different range in between leaves nothing behind that matters
    other = _records(torch, ps, lib.ps_scan_device_noalloc, g, 150, 160)
    np.testing.assert_allclose(other, _records(torch, ps, lib.ps_scan_device, g, 150, 160), rtol=1e-12, atol=0)
    again = _records(torch, ps, lib.ps_scan_device_noalloc, g, 11, 40)
    np.testing.assert_allclose(again, ref, rtol=1e-12, atol=0)
    g.close()


def test_noalloc_on_caller_stream_right_after_setup(native):
    """A caller's own stream, used straight after ps_set_conw_r returns: the
    scan must see the tables that call uploaded (no ordering with the
    context's internal stream is needed)."""
    torch = pytest.importorskip("torch")
    ps = native
    lib = ps.load_library()
    g = ps.PeriodSearch(golden_path("c1"))
    g.set_conw_r(g.conw_r * 8)
    ref = _records(torch, ps, lib.ps_scan_device, g, 11, 40)
    g.close()
    s = torch.cuda.Stream()
    for _ in range(2):
        g = ps.PeriodSearch(golden_path("c1"))
        g.set_conw_r(g.conw_r * 8)
        got = _records(torch, ps, lib.ps_scan_device_noalloc, g, 11, 40, ctypes.c_void_p(s.cuda_stream))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
        g.close()


def test_noalloc_rejects_oversized_request(native, tmp_path):
    torch = pytest.importorskip("torch")
    ps = native
    lib = ps.load_library()
    # the tiny asteroid over 2-100 h at a fine step: ~690 000 trial periods,
    # whose per-fit results alone (72 B x 10 fits each) exceed 64 MiB
    text = open(golden_path("tiny")).read().split("\n", 1)
    path = tmp_path / "period_search_in"
    path.write_text("2.0 0.05 100.0 1 fine scan\n" + text[1])
    g = ps.PeriodSearch(str(path))
    g.set_conw_r(g.conw_r)
    assert g.n_periods > 100000
    d = torch.zeros(g.n_periods * 6, dtype=torch.float64, device="cuda")  # sized for the range asked
    rc = lib.ps_scan_device_noalloc(g._h, 1, g.n_periods, ctypes.c_void_p(d.data_ptr()), None)
    assert rc == ps.PS_ERR_LIMIT
    assert b"64 MiB" in lib.ps_last_error()
    g.close()
