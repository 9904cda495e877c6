"""Per-exposure weight preprocessing (updc/_engine.py:287-408 of the reference).

CPU: the oracle's restatement against the golden outputs of the reference's
own functions (tests/golden/preprocess/, make_preprocess_golden.py) and its
float32 standard deviation against NumPy.  GPU: the library's preprocessing
(``updc_b200.preprocess``) against the golden outputs — same files, metrics,
log lines and error messages — and against the oracle on larger seeded
exposures (bit-identical WHT, sky mask and metrics).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import preprocess as OP
from updc_b200 import synth

GOLDEN = Path(__file__).parent / "golden" / "preprocess"


def _expected():
    return json.loads((GOLDEN / "expected.json").read_text())


def _paths(name, n):
    return [Path(f"/data/{name}_{i}_cal.fits") for i in range(1, n + 1)]


def _reader(path: Path):
    stem = path.name[: -len("_cal.fits")]
    name, index = stem.rsplit("_", 1)
    return synth.preprocess_case(name, int(index))


@pytest.mark.parametrize("n", [1, 7, 8, 9, 127, 128, 129, 1000, 8193, 65537, 300001])
def test_std_restatement_matches_numpy(n):
    rng = np.random.default_rng(n)
    a = (rng.standard_normal(n) * 3.0 + 1.0).astype(np.float32)
    assert OP.std_f32(a) == np.std(a)
    assert OP.median(a) == np.median(a)


def test_oracle_matches_reference_golden():
    exp = _expected()
    wht = np.load(GOLDEN / "wht.npz")
    for name, case in exp["cases"].items():
        _shape, mode, dqm, ped, _ = synth.PREPROCESS_CASES[name]
        for i, path in enumerate(_paths(name, case["exposures"]), 1):
            d = synth.preprocess_case(name, i)
            args = (d["SCI"], d["DQ"], d["VAR_POISSON"], d["VAR_RNOISE"], d["VAR_FLAT"], mode, dqm, ped, str(path))
            if "error" in case:
                with pytest.raises(ValueError) as err:
                    OP.prepare_exposure(*args)
                assert str(err.value) == case["error"], name
                continue
            w, m, _passes, _fb = OP.prepare_exposure(*args)
            assert np.array_equal(w, wht[f"{name}_{i}"]), name
            ref = case["metrics"][i - 1]
            for k, v in m.items():
                assert ref[k] == v, (name, k, ref[k], v)


def test_golden_covers_every_branch():
    exp = _expected()["cases"]
    errors = {c["error"].split(" in /")[0] for c in exp.values() if "error" in c}
    assert errors == {"Too few valid pixels for robust background estimation",
                      "Cannot estimate a positive background RMS", "Cannot estimate sky VAR_POISSON",
                      "No usable pixels remain", "Automatic pedestal failed to make y_eff positive",
                      "inverse-variance"}
    assert {c["weight_mode"] for c in exp.values() if "metrics" in c} == {"mask", "rnoise-sky", "totalvar"}
    d = synth.preprocess_case("mad_zero")
    *_, fallbacks = OP.prepare_exposure(d["SCI"], d["DQ"], d["VAR_POISSON"], d["VAR_RNOISE"], d["VAR_FLAT"],
                                        "rnoise-sky", 1, 0.0)
    assert fallbacks > 0


# ----------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_gpu_prepare_weighted_inputs_matches_reference_golden(engine_lib, tmp_path, capsys):
    from updc_b200 import preprocess as P
    exp = _expected()
    for name, case in exp["cases"].items():
        shape, mode, dqm, ped, _ = synth.PREPROCESS_CASES[name]
        out = tmp_path / name
        out.mkdir()
        images = _paths(name, case["exposures"])
        if "error" in case:
            with pytest.raises(ValueError) as err:
                P.prepare_weighted_inputs(images, out, mode, dqm, ped, shape, 1, read_planes=_reader)
            assert str(err.value) == case["error"], name
            continue
        capsys.readouterr()
        prepared, metrics = P.prepare_weighted_inputs(images, out, mode, dqm, ped, shape, 2, read_planes=_reader)
        assert capsys.readouterr().out.splitlines() == case["log"], name
        assert metrics == case["metrics"], name
        for (s, w), (sn, ssha, wn, wsha) in zip(prepared, case["files"]):
            assert (s.name, w.name) == (sn, wn)
            assert hashlib.sha256(s.read_bytes()).hexdigest() == ssha
            assert hashlib.sha256(w.read_bytes()).hexdigest() == wsha, name


def _big_case(shape, seed, pattern="sources"):
    d = synth.level2_exposure(shape, pattern, seed)
    return d["SCI"], d["DQ"], d["VAR_POISSON"].astype(np.float64), d["VAR_RNOISE"], d["VAR_FLAT"].astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,pattern,mode,ped", [
    ((512, 512), "sources", "rnoise-sky", 0.0),
    ((384, 640), "negative", "totalvar", 2.0),
    ((300, 300), "mad_zero", "rnoise-sky", 0.0),
    ((257, 263), "ties", "mask", 1.0),
    ((2048, 2048), "sources", "rnoise-sky", 0.0),
])
def test_gpu_matches_oracle(engine_lib, shape, pattern, mode, ped):
    from updc_b200 import preprocess as P
    planes = _big_case(shape, 7 + shape[0], pattern)
    w_ref, m_ref, passes, fallbacks = OP.prepare_exposure(*planes, mode, 1, ped, "x")
    w, m, sky = P.prepare_exposure(*planes, mode, 1, ped, "x", sky_mask=True)
    assert np.array_equal(w, w_ref)
    assert (m.pop("clip_passes"), m.pop("std_fallbacks")) == (passes, fallbacks)
    assert m == m_ref
    sci, dq, vp, vr, vf = planes
    base = np.isfinite(sci) & ((dq & 1) == 0) & np.isfinite(vp) & np.isfinite(vr)
    if mode == "totalvar":
        base &= np.isfinite(vf)
    mask, *_ = OP.robust_background(sci, base)
    assert np.array_equal(sky, mask)
    if pattern == "mad_zero":
        assert fallbacks > 0


@pytest.mark.gpu
def test_gpu_robust_background_mask(engine_lib):
    from updc_b200 import preprocess as P
    sci, dq, *_ = _big_case((640, 480), 11)
    base = np.isfinite(sci) & (dq == 0)
    for it in (1, 2, 6):
        mask, bg, sig = P.robust_background_mask(sci, base, it)
        rmask, rbg, rsig, *_ = OP.robust_background(sci, base, it)
        assert np.array_equal(mask, rmask) and bg == rbg and sig == rsig


@pytest.mark.gpu
def test_gpu_device_tensors_match_host_arrays(engine_lib):
    import torch
    from updc_b200 import preprocess as P
    planes = _big_case((400, 500), 21)
    w, m, sky = P.prepare_exposure(*planes, "totalvar", 1, 1.5, "x", sky_mask=True)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in planes]
    dev[1] = dev[1].view(torch.int32)
    wd, md, skyd = P.prepare_exposure(*dev, "totalvar", 1, 1.5, "x", sky_mask=True)
    torch.cuda.synchronize()
    assert np.array_equal(wd.cpu().numpy(), w) and np.array_equal(skyd.cpu().numpy(), sky) and md == m
