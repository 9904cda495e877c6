"""Engine-handoff formats (manifest, argv, synthetic inputs) on CPU."""
from __future__ import annotations

import numpy as np
import pytest

from updc_b200 import handoff, synth


def test_manifest_round_trip(tmp_path):
    rows = [handoff.ExposureRow(f"/d/sci_{k}.f32", f"/d/wht_{k}.f32", f"/d/psf_{k}.f32", 33, 31,
                                f"/d/v_{k}.bin", 0.1 * k + 0.3, 10.0 + k) for k in range(3)]
    m = tmp_path / "manifest.txt"
    handoff.write_manifest(m, rows)
    back = handoff.read_manifest(m, 3)
    assert back == rows
    assert back[1].links == "/d/v_1.bin.links"
    assert m.read_text().splitlines()[0].split("\t")[6] == "0.29999999999999999"


@pytest.mark.parametrize("mutate,msg", [
    (lambda rows: rows[:1], "fewer rows"),
    (lambda rows: rows + rows[:1], "more rows"),
])
def test_manifest_row_count_errors(tmp_path, mutate, msg):
    rows = [handoff.ExposureRow("s", "w", "p", 3, 3, "v", 0.3, 10.0) for _ in range(2)]
    m = tmp_path / "m.txt"
    handoff.write_manifest(m, mutate(rows))
    with pytest.raises(ValueError, match=msg):
        handoff.read_manifest(m, 2)


def test_manifest_value_errors(tmp_path):
    m = tmp_path / "m.txt"
    m.write_text("s\tw\tp\t0\t3\tv\t0.3\t10\n")
    with pytest.raises(ValueError, match="invalid PSF dimensions"):
        handoff.read_manifest(m, 1)
    m.write_text("s\tw\tp\t3\t3\tv\t0.3\t-1\n")
    with pytest.raises(ValueError, match="invalid background/pedestal"):
        handoff.read_manifest(m, 1)
    m.write_text("s\tw\tp\t3\n")
    with pytest.raises(ValueError, match="manifest requires"):
        handoff.read_manifest(m, 1)


def test_engine_args_order():
    a = handoff.EngineArgs("m", 10, 11, 5, 6, 2, 0, 3, "pre", "wht.bin", save_every=1)
    assert a.argv() == ["m", "10", "11", "5", "6", "2", "0", "3", "pre", "wht.bin", "1", "1", "1",
                        "0", "0", "0", "", "1"]


def test_synthetic_inputs_deterministic_and_valid(tmp_path):
    a = synth.generate("small", tmp_path / "a")
    b = synth.generate("small", tmp_path / "b")
    w = a.workload
    for ra, rb in zip(a.rows, b.rows):
        for f in ("science", "weight", "psf", "vertices"):
            assert open(getattr(ra, f), "rb").read() == open(getattr(rb, f), "rb").read()
        sci = np.fromfile(ra.science, np.float32)
        wht = np.fromfile(ra.weight, np.float32)
        psf = np.fromfile(ra.psf, np.float32)
        v = np.fromfile(ra.vertices, np.float64)
        assert sci.size == wht.size == w.iw * w.ih
        assert v.size == 2 * (w.iw + 1) * (w.ih + 1)
        assert abs(psf.astype(np.float64).sum() - 1.0) < 1e-5
        ok = np.isfinite(sci) & (wht > 0)
        assert np.all(sci[ok] + np.float32(ra.pedestal) > 0)
        assert np.isnan(sci).sum() >= 1
    assert handoff.read_manifest(a.manifest, w.nexp)[0].background == pytest.approx(0.3)


def test_workload_shapes():
    c1 = synth.WORKLOADS["c1"]
    assert (c1.W, c1.H, c1.iw, c1.ih, c1.nexp, c1.psf_size, c1.iterations) == (4096, 4096, 2048, 2048, 8, 1431, 39)
    c0 = synth.WORKLOADS["c0"]
    assert (c0.W, c0.iw, c0.nexp, c0.psf_size, c0.iterations) == (256, 128, 4, 33, 20)
