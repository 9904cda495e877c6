"""GPU PSF projector against the reference projector (psf_projector.c).

The reference projector is compiled unmodified from the reference sources
(oracle/Makefile); both executables get the same manifest of oversampled
PSFs with distorted corner maps, and the projected PSF files and the results
CSV must be byte-identical.
"""
from __future__ import annotations

import filecmp
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

CASES = [("p33", 33, 2, 1), ("p65", 65, 4, 2), ("p101", 101, 3, 3), ("p129", 129, 4, 4)]


def _manifest(tmp_path, tag):
    from updc_b200 import synth
    lines = []
    for name, size, over, seed in CASES:
        psf, vert = synth.psf_projection_case(tmp_path, name, size, over, seed)
        lines.append(f"{psf}\t{size}\t{size}\t{vert}\t{tmp_path / f'{name}.{tag}.f32'}\t{name}")
    m = tmp_path / f"manifest_{tag}.txt"
    m.write_text("\n".join(lines) + "\n")
    return m


@pytest.fixture(scope="module")
def reference_projector():
    if not O.REF_PROJECTOR.is_file():
        if (O.REFERENCE_SOURCES / "psf_projector.c").is_file():
            O.build(reference=True)
    if not O.REF_PROJECTOR.is_file():
        pytest.skip("reference projector not built (reference sources absent)")
    return O.REF_PROJECTOR


def test_reference_projector_self_test(reference_projector):
    r = subprocess.run([str(reference_projector), "--self-test"], capture_output=True, text=True)
    assert r.returncode == 0 and "self-test: OK" in r.stdout


@pytest.mark.gpu
def test_gpu_projector_byte_identical(engine_lib, reference_projector, tmp_path):
    from updc_b200 import _lib
    exe = _lib.LIB_PATH.parent / "bin" / "updc_psf_projector"
    ref = subprocess.run([str(reference_projector), str(_manifest(tmp_path, "ref")), "4", str(tmp_path / "ref.csv")],
                         capture_output=True, text=True)
    assert ref.returncode == 0, ref.stderr
    ours = subprocess.run([str(exe), str(_manifest(tmp_path, "gpu")), "4", str(tmp_path / "gpu.csv")],
                          capture_output=True, text=True)
    assert ours.returncode == 0, ours.stderr
    for name, *_ in CASES:
        assert filecmp.cmp(tmp_path / f"{name}.ref.f32", tmp_path / f"{name}.gpu.f32", shallow=False), name
    assert (tmp_path / "ref.csv").read_text() == (tmp_path / "gpu.csv").read_text()
    out = np.fromfile(tmp_path / "p65.gpu.f32", np.float32)
    assert abs(out.sum() - 1.0) < 1e-4


@pytest.mark.gpu
def test_gpu_projector_rejects_like_the_reference(engine_lib, reference_projector, tmp_path):
    from updc_b200 import _lib, synth
    exe = _lib.LIB_PATH.parent / "bin" / "updc_psf_projector"
    psf, vert = synth.psf_projection_case(tmp_path, "bad", 33, 2, 9)
    a = np.fromfile(psf, np.float32)
    a[5] = -1.0
    a.tofile(psf)
    (tmp_path / "m.txt").write_text(f"{psf}\t33\t33\t{vert}\t{tmp_path / 'o.f32'}\tbad\n")
    ref = subprocess.run([str(reference_projector), str(tmp_path / "m.txt"), "1", str(tmp_path / "r.csv")],
                         capture_output=True, text=True)
    ours = subprocess.run([str(exe), str(tmp_path / "m.txt"), "1", str(tmp_path / "g.csv")],
                          capture_output=True, text=True)
    assert ref.returncode == ours.returncode == 1
    assert ours.stderr.strip() == ref.stderr.strip() == "UPDC_PSF_PROJECT: PSF contains negative/non-finite pixels"


@pytest.mark.parametrize("text", [
    "",                                             # empty
    "# only a comment\n\n",                         # comments and blank lines only
    "a.f32\t33\t33\tv.bin\n",                       # too few fields
    "a.f32\t0\t33\tv.bin\to.f32\tlabel\n",          # invalid dimensions
    "a.f32\t33\t-2\tv.bin\to.f32\tlabel\n",
    "x" * 1100 + "\t33\t33\tv.bin\to.f32\tlabel\n",  # path too long
    "\r\n",                                         # a CR-only line is a row without fields
])
def test_projector_manifest_errors_like_the_reference(engine_lib, reference_projector, tmp_path, text):
    """Manifest rows the projectors reject before any projection (no GPU work):
    the same message and exit status as the reference projector."""
    from updc_b200 import _lib
    exe = _lib.LIB_PATH.parent / "bin" / "updc_psf_projector"
    m = tmp_path / "m.txt"
    m.write_text(text)
    ref = subprocess.run([str(reference_projector), str(m), "1", str(tmp_path / "r.csv")],
                         capture_output=True, text=True)
    ours = subprocess.run([str(exe), str(m), "1", str(tmp_path / "g.csv")], capture_output=True, text=True)
    assert ref.returncode == ours.returncode == 1
    assert ours.stderr == ref.stderr
