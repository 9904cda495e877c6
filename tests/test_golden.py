"""Golden fixtures written by the reference core (tests/golden/make_golden.py).

CPU: the oracle reproduces them bit for bit (x after every iteration, freeze
rows, LinkMap bytes).  GPU: the engine's LinkMaps are byte-identical, its WHT
product bit-identical, its freeze rows identical and x within 1e-5 relative
RMS after every iteration.
"""
from __future__ import annotations

import csv
import filecmp
import json
import shutil
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_rms

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["small", "small_forced_freeze"]


def _stage(case: str, tmp: Path):
    """Copy a case to tmp with an absolute-path manifest; returns (meta, manifest)."""
    src = GOLDEN / case
    meta = json.loads((src / "meta.json").read_text())
    for f in src.iterdir():
        shutil.copy(f, tmp / f.name)
    from updc_b200 import handoff
    rows = handoff.read_manifest(tmp / "manifest.txt", meta["nexp"])
    for r in rows:
        for field in ("science", "weight", "psf", "vertices"):
            setattr(r, field, str(tmp / getattr(r, field)))
    handoff.write_manifest(tmp / "manifest.txt", rows)
    return meta, tmp / "manifest.txt", rows


def _golden_rows(tmp: Path):
    with open(tmp / "ref_mufreeze.csv") as f:
        return [(int(r["n_new_frozen"]), int(r["n_total_frozen"]), r["min_raw_mu"]) for r in csv.DictReader(f)]


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_golden(oracle, case, tmp_path):
    meta, manifest, rows = _stage(case, tmp_path)
    W, H, iw, ih, n, its = (meta[k] for k in ("W", "H", "iw", "ih", "nexp", "iterations"))
    for k, row in enumerate(rows):
        out = tmp_path / f"orc_{k}.links"
        oracle.linkmap_build(row.vertices, iw, ih, W, H, str(out))
        assert filecmp.cmp(out, row.links, shallow=False)
    fw, fh = meta["fft_shape_reference"]
    s = oracle.Solver(str(manifest), W, H, iw, ih, n, fw, fh, precision=32)
    mine = []
    for it in range(1, its + 1):
        new, tot, mn = s.iterate(1)
        ref = np.fromfile(tmp_path / f"ref_{it:02d}.bin", np.float32).reshape(H, W)
        np.testing.assert_array_equal(s.estimate, ref)
        mine += [(int(new[0, k]), int(tot[0, k]), f"{np.float32(mn[0, k]):.9g}") for k in range(n)]
    assert mine == _golden_rows(tmp_path)
    wht = (s.coverage * np.float32(s.weight_scale)).astype(np.float32)
    np.testing.assert_array_equal(wht.reshape(-1), np.fromfile(tmp_path / "ref_wht.bin", np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("form", ["fp32", "fp32-reference"])
def test_engine_matches_golden(engine_lib, oracle, case, form, tmp_path):
    """x within 1e-5 relative RMS of the reference after every iteration.  The
    forced-FreezeMu case is ill-conditioned (ratios y/raw_mu with raw_mu close
    to 0 after cancellation against the -100 background): there even the exact
    FP64 oracle drifts from the FP32 reference by ~5e-5 after one iteration and
    ~1e-2 after four.  For it both FP32 solvers are compared with the FP64
    oracle: the engine's error must stay within 20x the reference core's own
    FP32 error (floor 1e-5)."""
    from updc_b200.engine import Engine
    meta, manifest, rows = _stage(case, tmp_path)
    W, H, iw, ih, n, its = (meta[k] for k in ("W", "H", "iw", "ih", "nexp", "iterations"))
    fw, fh = meta["fft_shape_reference"]
    s64 = oracle.Solver(str(manifest), W, H, iw, ih, n, fw, fh, precision=64)
    golden_links = []
    for row in rows:
        p = Path(row.links)
        golden_links.append(p.read_bytes())
        p.unlink()  # the engine must rebuild them on the GPU
    e = Engine(form=form)
    e.load(str(manifest), W, H, iw, ih, n)
    e.setup()
    for row, gold in zip(rows, golden_links):
        assert Path(row.links).read_bytes() == gold
    wht = (e.plane("coverage") * np.float32(e.weight_scale)).astype(np.float32)
    np.testing.assert_array_equal(wht.reshape(-1), np.fromfile(tmp_path / "ref_wht.bin", np.float32))
    mine = []
    for it in range(1, its + 1):
        st = e.iterate(1)[0]
        s64.iterate(1)
        ref = np.fromfile(tmp_path / f"ref_{it:02d}.bin", np.float32).reshape(H, W)
        if meta["background_override"] is None:
            assert rel_rms(e.plane("estimate"), ref) <= 1e-5, it
        else:
            ref_err = rel_rms(ref, s64.estimate)
            ours = rel_rms(e.plane("estimate"), s64.estimate)
            assert ours <= max(1e-5, 20.0 * ref_err), (it, ours, ref_err)
        mine += [(int(st.new_frozen[k]), int(st.total_frozen[k])) for k in range(n)]
    assert mine == [(a, b) for a, b, _ in _golden_rows(tmp_path)]
