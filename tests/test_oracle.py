"""The oracle itself, pinned against the compiled reference core and numpy (CPU)."""
from __future__ import annotations

import csv
import filecmp
import subprocess

import numpy as np
import pytest

from conftest import fft_shape_for


def _run_ref(ref_bin, ds, iterations, prefix):
    r = subprocess.run([str(ref_bin), *ds.engine_args(iterations=iterations, prefix=prefix).argv()],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    w = ds.workload
    x = np.fromfile(f"{ds.directory}/{prefix}_{iterations:02d}.bin", np.float32).reshape(w.H, w.W)
    with open(f"{ds.directory}/{prefix}_mufreeze.csv") as f:
        rows = list(csv.DictReader(f))
    return x, rows


def test_reference_self_test(reference_binary):
    r = subprocess.run([str(reference_binary), "--self-test"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK" in r.stdout


@pytest.mark.parametrize("name,background", [("small", None), ("abs32", None), ("abs32_wide", None),
                                             ("c0", None), ("c0", -100.0)])
def test_oracle_fp32_bit_exact_with_reference(reference_binary, oracle, datasets, name, background):
    """The FP32 restatement reproduces the reference core bit for bit: LinkMap
    bytes, x after every iteration of the workload, and every freeze CSV row."""
    ds = datasets(name, background)
    w = ds.workload
    iters = w.iterations if background is None else 3
    xref, rows = _run_ref(reference_binary, ds, iters, "pin")
    encs = []
    for k, row in enumerate(ds.rows):
        out = f"{row.vertices}.orc"
        nl, enc = oracle.linkmap_build(row.vertices, w.iw, w.ih, w.W, w.H, out)
        assert filecmp.cmp(row.links, out, shallow=False)
        encs.append(enc)
    if name.startswith("abs32"):
        assert set(encs) == {1}
    else:
        assert set(encs) == {2}
    pw, ph = ds.rows[0].psf_width, ds.rows[0].psf_height
    fw, fh = oracle.next_fast_size(w.W + pw - 1), oracle.next_fast_size(w.H + ph - 1)
    s = oracle.Solver(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=32)
    new, tot, mn = s.iterate(iters)
    np.testing.assert_array_equal(s.estimate, xref)
    mine = [(int(new[i, k]), int(tot[i, k]), f"{np.float32(mn[i, k]):.9g}")
            for i in range(iters) for k in range(w.nexp)]
    theirs = [(int(r["n_new_frozen"]), int(r["n_total_frozen"]), f"{float(r['min_raw_mu']):.9g}") for r in rows]
    assert mine == theirs
    if background is not None:
        assert tot[-1].sum() > 0


def test_fp64_oracle_close_to_reference(reference_binary, oracle, datasets):
    """The FP64 oracle and the FP32 reference agree to FP32 accuracy (c0, 20 iterations)."""
    ds = datasets("c0")
    w = ds.workload
    xref, _ = _run_ref(reference_binary, ds, w.iterations, "pin64")
    fw, fh = fft_shape_for(ds)
    s = oracle.Solver(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=64)
    s.iterate(w.iterations)
    d = s.estimate - xref
    assert np.sqrt(np.mean(d ** 2) / np.mean(xref.astype(np.float64) ** 2)) < 2e-5


@pytest.mark.parametrize("shape", [(12, 10), (9, 15), (35, 48), (288, 288), (96, 112)])
def test_shim_fft_matches_numpy(oracle, shape):
    """The FFTW-API shim (the reference core's FFT here) against numpy's FP64 FFT."""
    import ctypes
    L = ctypes.CDLL(str(oracle.SHIM_PATH))
    L.fftwf_plan_dft_r2c_2d.restype = ctypes.c_void_p
    L.fftwf_plan_dft_r2c_2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint]
    L.fftwf_plan_dft_c2r_2d.restype = ctypes.c_void_p
    L.fftwf_plan_dft_c2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint]
    L.fftwf_execute_dft_r2c.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.fftwf_execute_dft_c2r.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.fftwf_destroy_plan.argtypes = [ctypes.c_void_p]
    n0, n1 = shape
    rng = np.random.default_rng(n0 * 1000 + n1)
    x = rng.standard_normal((n0, n1)).astype(np.float32)
    X = np.zeros((n0, n1 // 2 + 1), np.complex64)
    p = L.fftwf_plan_dft_r2c_2d(n0, n1, x.ctypes.data, X.ctypes.data, 0)
    L.fftwf_execute_dft_r2c(p, x.ctypes.data, X.ctypes.data)
    ref = np.fft.rfft2(x.astype(np.float64))
    assert np.abs(X - ref).max() <= 2e-6 * np.abs(ref).max()
    q = L.fftwf_plan_dft_c2r_2d(n0, n1, X.ctypes.data, x.ctypes.data, 0)
    Y = ref.astype(np.complex64)
    y = np.zeros((n0, n1), np.float32)
    L.fftwf_execute_dft_c2r(q, Y.ctypes.data, y.ctypes.data)
    refy = np.fft.irfft2(ref, s=(n0, n1)) * n0 * n1
    assert np.abs(y - refy).max() <= 2e-6 * np.abs(refy).max()
    L.fftwf_destroy_plan(p)
    L.fftwf_destroy_plan(q)


def test_oracle_geometry_known_answers(oracle):
    """The reference self-test's known answers (updc_core.c:1545-1557)."""
    unit = np.array([[1000.0, 2000.0], [1000.0, 2001.0], [1001.0, 2001.0], [1001.0, 2000.0]])
    assert abs(oracle.polygon_area(unit) - 1.0) <= 2e-6
    half = np.array([[-0.5, -0.5], [-0.5, 0.5], [0.0, 0.5], [0.0, -0.5]])
    assert abs(oracle.overlap_area(half, 0, 0) - 0.5) <= 2e-6


def test_next_fast_size(oracle):
    assert oracle.next_fast_size(5526) == 5600
    assert oracle.next_fast_size(9622) == 9720
    assert oracle.next_fast_size(3478) == 3500
    assert oracle.next_fast_size(288) == 288
