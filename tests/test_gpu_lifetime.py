"""Context lifetime with asynchronous scans (the per-device buffer cache).

ps_scan_device on a caller's stream returns before the scan has run; a
ps_close right after it must not hand the context's buffers to the next
context while the scan still reads them.  The test closes the context at
once, opens another asteroid (whose uploads draw from the same cache), and
checks that the first scan's records are those of an undisturbed scan."""
import ctypes

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def test_close_waits_for_a_scan_on_a_caller_stream(native):
    torch = pytest.importorskip("torch")
    ps = native
    g = ps.PeriodSearch(golden_path("c1"), form=ps.PS_FORM_FAST)
    g.set_conw_r(g.conw_r * 8)
    want = g.scan(1, 60)
    g.close()
    stream = torch.cuda.Stream()
    for _ in range(3):
        g = ps.PeriodSearch(golden_path("c1"), form=ps.PS_FORM_FAST)
        g.set_conw_r(g.conw_r * 8)
        d = torch.full((60 * 6,), float("nan"), dtype=torch.float64, device="cuda")
        g.scan_device(1, 60, d.data_ptr(), stream.cuda_stream)
        g.close()  # no synchronisation in between
        other = ps.PeriodSearch(golden_path("shipped"), form=ps.PS_FORM_FAST)
        other.set_conw_r(other.conw_r)
        other.scan(1, 4)
        torch.cuda.synchronize()
        got = d.view(60, 6).cpu().numpy()
        other.close()
        for k, name in enumerate(want.dtype.names):
            assert np.array_equal(got[:, k], want[name]), name
