"""FFT autotuner: candidate shapes and radix splits timed on the device,
cached like the reference's fft_autotune_v1 files (updc_core.c:195-291)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import crop_min_shape


@pytest.mark.gpu
def test_autotune_choice_cache_and_results(engine_lib, datasets, tmp_path):
    from updc_b200.engine import Engine
    ds = datasets("medium")
    w = ds.workload
    min_w, min_h = crop_min_shape(ds)   # shapes below these would change the kept window

    def run(**kw):
        e = Engine(form="fp32", **kw)
        e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
        return e

    tuned = run(autotune=True, tune_cache_dir=tmp_path)
    fw, fh = tuned.fft_shape
    assert fw % 2 == 0 and fw >= min_w and fh >= min_h
    assert int(np.prod(tuned.fft_radices(0))) == fw // 2
    assert int(np.prod(tuned.fft_radices(1))) == fh
    info = tuned.autotune_info
    assert info["plans_timed"] > 0 and not info["cache_hit"] and info["modelled_ms"] > 0
    assert list(tmp_path.glob("fft_autotune_b200_v1_f32_*.txt"))

    again = run(autotune=True, tune_cache_dir=tmp_path)
    assert again.autotune_info["cache_hit"] and again.autotune_info["plans_timed"] == 0
    assert again.fft_shape == (fw, fh)
    assert again.fft_radices(0) == tuned.fft_radices(0) and again.fft_radices(1) == tuned.fft_radices(1)
    again.close()

    retuned = run(autotune=True, retune=True, tune_cache_dir=tmp_path)
    assert not retuned.autotune_info["cache_hit"] and retuned.autotune_info["plans_timed"] > 0
    retuned.close()

    # a different padded shape / radix split only changes rounding
    plain = run()
    tuned.iterate(w.iterations)
    plain.iterate(w.iterations)
    a, b = tuned.plane("estimate", as_double=True), plain.plane("estimate", as_double=True)
    rel = float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))
    assert rel <= 1e-5, rel
    tuned.close()
    plain.close()
