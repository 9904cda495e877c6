"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    """The oracle library (built on demand; test infrastructure only)."""
    from oracle import oracle as O
    if not O.LIB_PATH.is_file():
        O.build(reference=False)
    O.lib()
    return O


@pytest.fixture(scope="session")
def reference_binary(oracle):
    """The reference core compiled from its sources with the FFTW-API shim."""
    if not oracle.REF_BINARY.is_file():
        if oracle.REFERENCE_SOURCES.is_dir():
            oracle.build(reference=True)
    if not oracle.REF_BINARY.is_file():
        pytest.skip("reference core binary not built (reference sources absent)")
    return oracle.REF_BINARY


@pytest.fixture(scope="session")
def engine_lib():
    """The B200 engine library (built in-tree on demand; nvcc cross-compiles)."""
    from updc_b200 import _lib, build
    if not _lib.LIB_PATH.is_file() or not _lib.EXE_PATH.is_file():
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def datasets(tmp_path_factory):
    """Factory of synthetic handoff datasets, generated once per session."""
    from updc_b200 import synth
    cache = {}

    def get(name: str, background=None):
        key = (name, background)
        if key not in cache:
            d = tmp_path_factory.mktemp(f"data_{name}")
            ds = synth.generate(name, d)
            if background is not None:
                from updc_b200 import handoff
                for r in ds.rows:
                    r.background = background
                handoff.write_manifest(ds.manifest, ds.rows)
            cache[key] = ds
        return cache[key]

    return get


def fft_shape_for(ds, even_width: bool = True):
    """The FFT shape the engine picks (smallest even/any 7-smooth sizes)."""
    from oracle import oracle as O
    w = ds.workload
    pw = max(r.psf_width for r in ds.rows)
    ph = max(r.psf_height for r in ds.rows)
    fw = O.next_fast_size(w.W + pw - 1)
    while even_width and fw % 2:
        fw = O.next_fast_size(fw + 1)
    return fw, O.next_fast_size(w.H + ph - 1)


def crop_min_shape(ds, transposed: bool = False):
    """Smallest circular lengths whose kept W x H window is exactly the linear
    convolution's: n + f/2 per axis (and at least f), with f the largest PSF
    extent along that axis."""
    w = ds.workload
    pw = max(r.psf_width for r in ds.rows)
    ph = max(r.psf_height for r in ds.rows)
    if transposed:
        pw, ph = ph, pw
    return max(w.W + pw // 2, pw), max(w.H + ph // 2, ph)


def rel_rms(a, b):
    import numpy as np
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / max(np.mean(b ** 2), 1e-300)))
