"""Whole-solve parity with the reference core on the handoff's remaining cases.

* the headline workload (c1: 8 x 2048^2 detectors -> 4096^2, 1431^2 PSFs,
  39 iterations) against the reference core compiled from its own sources
  (oracle/_ref), run on this machine's host cores on the same files;
* the transposed-PSF handoff (psf_transposed = 1, updc/_engine.py:1384):
  non-square, asymmetric PSFs, forward model against the FP64 oracle and a
  whole solve against the reference core;
* the Kahan-compensated FP32 form against the FP64 oracle.
"""
from __future__ import annotations

import csv
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu


def _reference(ref_bin, ds, iterations, prefix, transposed=0, timeout=1800):
    """Runs the reference core on a dataset; returns (x, freeze rows)."""
    w = ds.workload
    cores = os.cpu_count() or 1
    a = ds.engine_args(iterations=iterations, prefix=prefix, fft_workers=max(1, cores // w.nexp),
                       exposure_workers=w.nexp, preprocess_workers=w.nexp)
    a.psf_transposed = transposed
    r = subprocess.run([str(ref_bin), *a.argv()], capture_output=True, text=True, timeout=timeout,
                       env={**os.environ, "UPDC_PERSIST_CACHE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    x = np.fromfile(f"{ds.directory}/{prefix}_{iterations:02d}.bin", np.float32).reshape(w.H, w.W)
    with open(f"{ds.directory}/{prefix}_mufreeze.csv") as f:
        rows = list(csv.DictReader(f))
    return x, rows


def _solve(ds, form, iterations, transposed=0, **kw):
    from updc_b200.engine import Engine
    w = ds.workload
    e = Engine(form=form, **kw)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, transposed)
    e.setup()
    st = e.iterate(iterations, check_each=False)
    x = e.plane("estimate")
    rows = [(int(s.new_frozen[k]), int(s.total_frozen[k]), float(s.min_raw_mu[k])) for s in st for k in range(w.nexp)]
    e.close()
    return x, rows


def _freeze_counts(rows):
    return [(int(r["n_new_frozen"]), int(r["n_total_frozen"])) for r in rows]


def test_c1_headline_matches_reference_core(engine_lib, reference_binary, tmp_path):
    """c1 after its 39 iterations: the FP32 form within 1e-5 relative RMS of
    the reference core's x, the per-iteration FreezeMu counts of both FP32
    forms equal to the reference's freeze CSV (updc_core.c:1425-1431), and the
    per-exposure min raw_mu within FFT rounding of the reference's."""
    from updc_b200 import synth
    ds = synth.generate("c1", tmp_path, use_torch=True)
    w = ds.workload
    # the engine runs first and writes the LinkMaps (byte-identical to the
    # reference's), which the reference then reuses under UPDC_PERSIST_CACHE
    x32, rows32 = _solve(ds, "fp32", w.iterations)
    xr32, rowsr32 = _solve(ds, "fp32-reference", w.iterations)
    xref, ref_rows = _reference(reference_binary, ds, w.iterations, "ref_c1")
    err32 = rel_rms(x32, xref)
    errr = rel_rms(xr32, xref)
    print(f"c1 rel RMS vs reference core: fp32 {err32:.3e}, fp32-reference {errr:.3e}")
    assert err32 <= 1e-5
    assert errr <= 2e-5
    counts = _freeze_counts(ref_rows)
    assert [(a, b) for a, b, _ in rows32] == counts
    assert [(a, b) for a, b, _ in rowsr32] == counts
    ref_min = np.array([float(r["min_raw_mu"]) for r in ref_rows])
    for rows in (rows32, rowsr32):
        mine = np.array([m for _, _, m in rows])
        np.testing.assert_allclose(mine, ref_min, rtol=1e-4)


def _asymmetric_psf_dataset(ds, tmp: Path, pw: int = 25, ph: int = 15):
    """The dataset with every PSF replaced by a non-square (pw x ph as stored),
    asymmetric one: an off-centre elliptical Gaussian on a linear ramp."""
    from updc_b200 import handoff
    rows = []
    yy, xx = np.indices((ph, pw), dtype=np.float64)
    for k, r in enumerate(ds.rows):
        psf = np.exp(-0.5 * (((xx - 0.35 * pw - k) / 2.6) ** 2 + ((yy - 0.6 * ph) / 1.3) ** 2))
        psf += 0.02 * (1.0 + xx / pw + 2.0 * yy / ph)
        p = tmp / f"psf_asym_{k}.f32"
        psf.astype(np.float32).tofile(p)
        rows.append(handoff.ExposureRow(**{**r.__dict__, "psf": str(p), "psf_width": pw, "psf_height": ph}))
    m = tmp / "manifest_asym.txt"
    handoff.write_manifest(m, rows)
    return m, rows


@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_transposed_psf_forward_model(engine_lib, oracle, datasets, form, tol, tmp_path):
    """psf_transposed = 1 with 25 x 15 stored PSFs: the forward extents are
    15 x 25 and pixel (x, y) is read at x*pw + y (updc_core.c:814-819).  The
    engine's forward model equals the FP64 oracle's; read untransposed it
    would not."""
    from updc_b200.engine import Engine
    ds = datasets("c0")
    w = ds.workload
    manifest, rows = _asymmetric_psf_dataset(ds, tmp_path)
    fw = w.W + 15 - 1                      # forward width = the stored height
    while fw % 2 or oracle.next_fast_size(fw) != fw:
        fw += 1
    fh = oracle.next_fast_size(w.H + 25 - 1)
    s64 = oracle.Solver(str(manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=64, transposed=1)
    e = Engine(form=form)
    e.load(str(manifest), w.W, w.H, w.iw, w.ih, w.nexp, 1)
    e.setup()
    e.set_plane("estimate", s64.estimate)
    e.stage_forward()
    plain = Engine(form=form)
    plain.load(str(manifest), w.W, w.H, w.iw, w.ih, w.nexp, 0)
    plain.setup()
    plain.set_plane("estimate", s64.estimate)
    plain.stage_forward()
    for k in range(w.nexp):
        ref = s64.forward_blur(k)
        assert rel_rms(e.plane("blur", k, as_double=True), ref) <= tol
        assert rel_rms(plain.plane("blur", k, as_double=True), ref) > 1e-3
    e.close()
    plain.close()


def test_transposed_psf_solve_matches_reference_core(engine_lib, reference_binary, datasets, tmp_path):
    """The whole c0 solve with transposed non-square PSFs: FP32 form within
    1e-5 relative RMS of the reference core given transpose_psf = 1, and the
    same FreezeMu counts."""
    from updc_b200 import handoff, synth
    ds = datasets("c0")
    manifest, rows = _asymmetric_psf_dataset(ds, tmp_path)
    ds2 = synth.Dataset(ds.workload, tmp_path, manifest, rows)
    xref, ref_rows = _reference(reference_binary, ds2, ds.workload.iterations, "ref_t", transposed=1)
    x, mine = _solve(ds2, "fp32", ds.workload.iterations, transposed=1)
    assert rel_rms(x, xref) <= 1e-5
    assert [(a, b) for a, b, _ in mine] == _freeze_counts(ref_rows)


def test_kahan_form_matches_fp64_oracle(engine_lib, oracle, datasets):
    """The Kahan-compensated FP32 form (FP32 products, compensated FP32
    cross-exposure sums, Kahan FP32 denominator) after the c0 solve's 20
    iterations within 1e-5 relative RMS of the FP64 oracle, like the default
    FP32 form."""
    from conftest import fft_shape_for
    ds = datasets("c0")
    w = ds.workload
    fw, fh = fft_shape_for(ds)
    s64 = oracle.Solver(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=64)
    s64.iterate(w.iterations)
    xk, _ = _solve(ds, "fp32-kahan", w.iterations)
    x32, _ = _solve(ds, "fp32", w.iterations)
    ek, e32 = rel_rms(xk, s64.estimate), rel_rms(x32, s64.estimate)
    print(f"c0 rel RMS vs FP64 oracle: fp32-kahan {ek:.3e}, fp32 {e32:.3e}")
    assert ek <= 1e-5
