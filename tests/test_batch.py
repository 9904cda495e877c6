"""Batched cutout fields: one persistent launch per stage over all fields.

CPU: the cutout generator follows the batched-field spec (grid sizes,
exposure counts, detector and PSF sizes).
GPU: every field of a batch ends bit-identical to the same field solved by
its own engine (same kernels' block bodies, same summation order), with the
same per-iteration signed sums and FreezeMu counts, for the whole-loop graph
and for checked single iterations.
"""
from __future__ import annotations

import numpy as np
import pytest


def test_batch_workloads_follow_the_spec():
    from updc_b200 import synth
    ws = synth.batch_workloads(64)
    assert len(ws) == 64
    for w in ws:
        assert w.W == w.H and w.W in synth.BATCH_GRIDS
        assert 3 <= w.nexp <= 12
        assert abs(w.iw - w.W // 2) <= 16 and w.iw == w.ih
        assert 33 <= w.psf_size <= 129 and w.psf_size % 2 == 1
        assert 1.0 <= w.psf_sigma <= 1.6
    assert synth.batch_workloads(64) == ws          # seeded


@pytest.fixture(scope="module")
def batch_data(tmp_path_factory):
    from updc_b200 import synth
    return synth.generate_batch(tmp_path_factory.mktemp("batch"), n_fields=6, seed=7, iterations=5)


def _single(ds, form):
    from updc_b200.engine import Engine
    w = ds.workload
    e = Engine(form=form)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    return e


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp32", "fp32-reference"])
def test_batch_matches_single_field_engines(engine_lib, batch_data, form):
    from updc_b200.batch import Batch
    b = Batch(form=form)
    for ds in batch_data:
        w = ds.workload
        b.add_field(ds.manifest, w.W, w.H, w.iw, w.ih, w.nexp)
    b.setup()
    assert b.units(1) == sum(b.field(i).fft_shape[0] // 2 + 1 for i in range(b.fields))
    recs = b.iterate(4, check_each=False) + b.iterate(1, check_each=True)
    singles = [_single(ds, form) for ds in batch_data]
    srecs = [e.iterate(5, check_each=True) for e in singles]
    for f, (ds, e) in enumerate(zip(batch_data, singles)):
        np.testing.assert_array_equal(b.field(f).plane("estimate"), e.plane("estimate"), err_msg=f"field {f}")
        for i in range(5):
            assert recs[i]["signed_sum"][f] == srecs[f][i].signed_sum
            assert recs[i]["negative"][f] == srecs[f][i].negative
    off = 0
    for f, ds in enumerate(batch_data):
        n = ds.workload.nexp
        for i in range(5):
            np.testing.assert_array_equal(recs[i]["total_frozen"][off:off + n], srecs[f][i].total_frozen)
        off += n
    assert all(r["seconds"] > 0 for r in recs)
    for e in singles:
        e.close()
    b.close()
