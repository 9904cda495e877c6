"""Regenerate the golden fixtures of the per-exposure weight preprocessing.

    python tests/golden/make_preprocess_golden.py

Runs the reference's own ``prepare_weighted_inputs`` (updc/_engine.py:336-408,
imported from the reference tree) on the synthetic Level-2 exposures of
``updc_b200.synth.PREPROCESS_CASES`` and writes what it produced to
tests/golden/preprocess/: for every case either the metrics records, the
printed log lines, the SHA-256 of the SCI/WHT raw files it wrote and the WHT
planes, or the message of the ValueError it raised.

The reference module imports astropy (absent here) at the top; only
``fits.open`` is reached on this path, so a stand-in module serves the
synthetic planes under the file names the reference opens.  NumPy's version is
recorded: the float32 rounding of the clipping thresholds and of the
standard-deviation fallback follows NumPy 2's promotion rules.
"""
from __future__ import annotations

import contextlib
import hashlib
import io
import json
import sys
import os
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
# the reference checkout: UPDC_REFERENCE_DIR, by default a sibling of this repository
REFERENCE = Path(os.environ.get("UPDC_REFERENCE_DIR", ROOT.parent / "reference"))
OUT = HERE / "preprocess"
sys.path.insert(0, str(ROOT))

from updc_b200 import synth  # noqa: E402

EXPOSURES = {"sky_sources": 3}
_PLANES: dict = {}


class _HDU:
    def __init__(self, data):
        self.data = data


class _HDUList:
    def __init__(self, planes):
        self._planes = planes

    def __contains__(self, name):
        return name in self._planes

    def __getitem__(self, name):
        return _HDU(self._planes[name])

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def _install_astropy_standin():
    fits = types.ModuleType("astropy.io.fits")
    fits.open = lambda path, memmap=False: _HDUList(_PLANES[str(path)])
    fits.Header = dict
    wcs = types.ModuleType("astropy.wcs")
    wcs.WCS = object
    io_mod = types.ModuleType("astropy.io")
    io_mod.fits = fits
    astropy = types.ModuleType("astropy")
    astropy.io, astropy.wcs = io_mod, wcs
    sys.modules.update({"astropy": astropy, "astropy.io": io_mod, "astropy.io.fits": fits, "astropy.wcs": wcs})


def sha256(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def main() -> None:
    _install_astropy_standin()
    sys.path.insert(0, str(REFERENCE))
    from updc import _engine as E  # the reference module

    OUT.mkdir(parents=True, exist_ok=True)
    record = {"numpy": np.__version__, "cases": {}}
    planes_out = {}
    for name, (shape, mode, dqmask, ped, _pattern) in synth.PREPROCESS_CASES.items():
        images = []
        for i in range(1, EXPOSURES.get(name, 1) + 1):
            path = Path(f"/data/{name}_{i}_cal.fits")
            _PLANES[str(path)] = synth.preprocess_case(name, i)
            images.append(path)
        with tempfile.TemporaryDirectory() as tmp:
            buf = io.StringIO()
            case = {"shape": list(shape), "weight_mode": mode, "bad_dq_mask": dqmask, "pedestal_sigma": ped,
                    "exposures": len(images)}
            try:
                with contextlib.redirect_stdout(buf):
                    prepared, metrics = E.prepare_weighted_inputs(images, Path(tmp), mode, dqmask, ped, shape, 1)
            except ValueError as exc:
                case["error"] = str(exc)
            else:
                case["metrics"] = metrics
                case["log"] = buf.getvalue().splitlines()
                case["files"] = [[Path(s).name, sha256(Path(s)), Path(w).name, sha256(Path(w))] for s, w in prepared]
                for i, (_s, w) in enumerate(prepared, 1):
                    planes_out[f"{name}_{i}"] = np.fromfile(w, dtype="<f4").reshape(shape)
        record["cases"][name] = case
        print(name, case.get("error", "ok"))
    (OUT / "expected.json").write_text(json.dumps(record, indent=1, sort_keys=True) + "\n")
    np.savez_compressed(OUT / "wht.npz", **planes_out)


if __name__ == "__main__":
    main()
