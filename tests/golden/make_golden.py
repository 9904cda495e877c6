"""Regenerate the golden fixtures from the reference core.

    python tests/golden/make_golden.py

Writes tests/golden/<case>/ for the small synthetic workload (normal and with
the manifest background forced to -100, the reference smoke test's FreezeMu
trigger, tests/test_smoke.py:116-121 in the reference): the engine-handoff
inputs, and the outputs of the reference core (updc/c_core/updc_core.c
compiled from its own sources with the FFTW-API shim, oracle/_ref) run with
save_every=1: x after every iteration, the freeze CSV, the WHT product and
the LinkMap v2 files it built.  Paths in the stored manifest are relative to
the case directory.
"""
from __future__ import annotations

import json
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from updc_b200 import handoff, synth  # noqa: E402

CASES = {"small": None, "small_forced_freeze": -100.0}


def make(case: str, background) -> None:
    out = HERE / case
    if out.exists():
        shutil.rmtree(out)
    out.mkdir(parents=True)
    with tempfile.TemporaryDirectory() as tmp:
        ds = synth.generate("small", tmp)
        rows = ds.rows
        if background is not None:
            for r in rows:
                r.background = background
            handoff.write_manifest(ds.manifest, rows)
        w = ds.workload
        args = ds.engine_args(iterations=w.iterations, prefix="ref", save_every=1).argv()
        r = O.run_reference(args)
        if r.returncode:
            raise SystemExit(r.stderr)
        rel_rows = []
        for k, row in enumerate(rows, 1):
            names = {}
            for field in ("science", "weight", "psf", "vertices"):
                src = Path(getattr(row, field))
                shutil.copy(src, out / src.name)
                names[field] = src.name
            shutil.copy(Path(row.links), out / f"{Path(row.vertices).name}.links")
            rel_rows.append(handoff.ExposureRow(names["science"], names["weight"], names["psf"], row.psf_width,
                                                row.psf_height, names["vertices"], row.background, row.pedestal))
        handoff.write_manifest(out / "manifest.txt", rel_rows)
        for it in range(1, w.iterations + 1):
            shutil.copy(Path(tmp) / f"ref_{it:02d}.bin", out / f"ref_{it:02d}.bin")
        shutil.copy(Path(tmp) / "ref_mufreeze.csv", out / "ref_mufreeze.csv")
        shutil.copy(Path(tmp) / "ref_wht.bin", out / "ref_wht.bin")
        meta = {"workload": "small", "W": w.W, "H": w.H, "iw": w.iw, "ih": w.ih, "nexp": w.nexp,
                "iterations": w.iterations, "background_override": background,
                "generator": "reference core (oracle/_ref) via tests/golden/make_golden.py",
                "fft_shape_reference": [O.next_fast_size(w.W + rows[0].psf_width - 1),
                                        O.next_fast_size(w.H + rows[0].psf_height - 1)]}
        (out / "meta.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    for case, bg in CASES.items():
        make(case, bg)
        print("wrote", HERE / case)
