"""updc_update_noalloc (file-scope scratch, no device allocation) against the
handle API's updc_stage_update on the same planes, two calls in a row.

Collected last (file name) so it also runs after every other test in the
same process; it passes on its own too.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _planes(e):
    return e.plane("correction"), e.plane("denominator"), e.plane("estimate")


def test_noalloc_update_matches_stage_update_twice(engine_lib, datasets):
    import torch
    from updc_b200.engine import Engine, update_noalloc

    ds = datasets("c0")
    w = ds.workload
    e = Engine(form="fp32", use_graph=False)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    ms = e.max_sensitivity
    stream = torch.cuda.Stream()
    for call in range(2):
        e.stage_forward()
        e.stage_detector()
        e.stage_correction()
        c, d, x = _planes(e)
        dc = torch.from_numpy(c).cuda()
        dd = torch.from_numpy(d).cuda()
        dx = torch.from_numpy(x).cuda()
        torch.cuda.synchronize()
        s_ref, n_ref = e.stage_update()            # existing entry point, engine-owned scratch
        x_ref = e.plane("estimate")
        s_new, n_new = update_noalloc(dc.data_ptr(), dd.data_ptr(), dx.data_ptr(), dx.numel(), ms,
                                      stream.cuda_stream)
        x_new = dx.cpu().numpy()
        # same kernels and grid on the same inputs: identical results
        np.testing.assert_array_equal(x_new, x_ref, err_msg=f"call {call + 1}")
        assert n_new == n_ref, f"call {call + 1}"
        assert s_new == pytest.approx(s_ref, rel=1e-12, abs=0.0), f"call {call + 1}"
    e.close()


def test_noalloc_update_rejects_sizes_and_reports_reference_errors(engine_lib):
    import torch
    from updc_b200 import _lib
    from updc_b200.engine import update_noalloc

    x = torch.ones(1024, device="cuda")
    d = torch.ones(1024, device="cuda")
    c = torch.ones(1024, device="cuda")
    with pytest.raises(_lib.UpdcError, match="exceeds the maximum"):
        update_noalloc(c.data_ptr(), d.data_ptr(), x.data_ptr(), (1 << 40) + 1, 1.0)
    with pytest.raises(_lib.UpdcError, match="empty plane"):
        update_noalloc(c.data_ptr(), d.data_ptr(), x.data_ptr(), 0, 1.0)
    # a substantially negative correction: the reference's message, and the
    # next call (error record re-armed) succeeds
    c[7] = -1.0
    with pytest.raises(_lib.UpdcError, match="substantially negative multiplicative correction"):
        update_noalloc(c.data_ptr(), d.data_ptr(), x.data_ptr(), 1024, 1.0)
    c[7] = 2.0
    x.fill_(1.0)
    s, neg = update_noalloc(c.data_ptr(), d.data_ptr(), x.data_ptr(), 1024, 1.0)
    assert neg == 0 and s == pytest.approx(1023.0 + 2.0)
