"""The C ABI library on CPU: it loads, exports every declared entry point, and its
host-side geometry matches the oracle bit for bit (no GPU calls)."""
from __future__ import annotations

import ctypes
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(engine_lib):
    from updc_b200 import _lib
    names = _lib.declared_functions()
    assert "UPDC_ALL" in names and "updc_create" in names and len(names) >= 25
    missing = [n for n in names if not hasattr(engine_lib, n)]
    assert not missing, missing


def test_version_and_errors_without_gpu(engine_lib):
    from updc_b200 import _lib
    assert b"sm_100a" in engine_lib.updc_version()
    opt = _lib.Options()
    engine_lib.updc_default_options(ctypes.byref(opt))
    assert opt.form == 0 and opt.use_graph == 1
    # invalid form is rejected before any device call
    opt.form = 9
    h = ctypes.c_void_p()
    assert engine_lib.updc_create(ctypes.byref(opt), ctypes.byref(h)) != 0
    assert b"precision form" in engine_lib.updc_last_error()


def test_host_geometry_bit_exact_with_oracle(engine_lib, oracle):
    """updc_polygon_area / updc_overlap_area (host build of the geometry the GPU
    LinkMap builder uses) against the oracle on random mapped pixels."""
    from updc_b200.engine import overlap_area, polygon_area
    rng = np.random.default_rng(7)
    for _ in range(2000):
        cx, cy = rng.uniform(-3, 3000, 2)
        th = rng.uniform(-0.3, 0.3)
        s = rng.uniform(0.5, 2.5)
        base = np.array([[-0.5, -0.5], [-0.5, 0.5], [0.5, 0.5], [0.5, -0.5]]) * s
        rot = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
        q = base @ rot.T + np.array([cx, cy]) + rng.normal(0, 0.05, (4, 2))
        assert np.float32(polygon_area(q)) == np.float32(oracle.polygon_area(q))
        tx, ty = int(round(cx)) + rng.integers(-1, 2), int(round(cy)) + rng.integers(-1, 2)
        assert np.float32(overlap_area(q, tx, ty)) == np.float32(oracle.overlap_area(q, tx, ty))


def test_dropin_usage_error(engine_lib):
    """Wrong argument count: the reference's usage message and exit status 1."""
    from updc_b200 import _lib
    r = subprocess.run([str(_lib.EXE_PATH), "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stderr.startswith("UPDC_ALL: usage: updc_jwst_c manifest")
