"""Engine-handoff file formats shared with the reference core.

The reference engine (updc/_engine.py:1300-1310, 1381-1390) hands the frozen
core a TSV manifest, raw little-endian float32 planes, float64 vertex maps and
18 positional arguments.  This module writes and reads exactly that contract so
the B200 engine is a drop-in for the same call:

* manifest: one row per exposure, 8 tab-separated fields
  ``science.f32 weight.f32 psf.f32 psf_w psf_h vertices.bin background pedestal``
  (updc/c_core/updc_core.c:426-461; written with ``%.17g`` at _engine.py:1305-1308);
* the LinkMap cache of exposure k is ``<vertices>.links`` (updc_core.c:452);
* vertices are ``(ih+1) x (iw+1) x 2`` float64 target-pixel coordinates of the
  detector pixel corners (_engine.py:272-280);
* argv: ``manifest W H iw ih nexp psf_transposed iterations prefix wht.bin
  fft_workers exposure_workers preprocess_workers plan_measure autotune
  retune_fft wisdom_path save_every`` (updc_core.c:1566-1572).
"""
from __future__ import annotations

import dataclasses
import os
from pathlib import Path
from typing import List, Sequence

# LinkMap v2 constants (updc/c_core/updc_core.c:44-54).
LINKMAP_MAGIC = 0x324D4C55  # "ULM2" little-endian
LINKMAP_VERSION = 2
LINKMAP_ENCODING_ABS32 = 1
LINKMAP_ENCODING_DELTA16 = 2
LINKMAP_HEADER_BYTES = 64


@dataclasses.dataclass
class ExposureRow:
    science: str
    weight: str
    psf: str
    psf_width: int
    psf_height: int
    vertices: str
    background: float
    pedestal: float

    @property
    def links(self) -> str:
        return self.vertices + ".links"

    def to_tsv(self) -> str:
        return (f"{self.science}\t{self.weight}\t{self.psf}\t{self.psf_width}\t{self.psf_height}\t"
                f"{self.vertices}\t{self.background:.17g}\t{self.pedestal:.17g}\n")


def write_manifest(path: os.PathLike, rows: Sequence[ExposureRow]) -> None:
    Path(path).write_text("".join(r.to_tsv() for r in rows))


def read_manifest(path: os.PathLike, exposures: int) -> List[ExposureRow]:
    """Parse a manifest with the reference's rules (updc_core.c:426-461).

    Raises ValueError with the reference's message on the same conditions:
    fewer or more rows than ``exposures``, missing fields, bad PSF sizes,
    non-finite background/pedestal or a negative pedestal.
    """
    import math
    lines = Path(path).read_text().splitlines(keepends=True)
    rows: List[ExposureRow] = []
    for k in range(exposures):
        if k >= len(lines):
            raise ValueError("manifest has fewer rows than expected")
        fields = [f for f in lines[k].replace("\r", "\t").replace("\n", "\t").split("\t") if f != ""]
        if len(fields) < 8:
            raise ValueError("manifest requires science, weight, psf, psf_width, psf_height, "
                             "vertices, background, pedestal")
        row = ExposureRow(fields[0], fields[1], fields[2], int(fields[3]), int(fields[4]),
                          fields[5], float(fields[6]), float(fields[7]))
        if row.psf_width < 1 or row.psf_height < 1:
            raise ValueError("invalid PSF dimensions in manifest")
        if (not math.isfinite(row.background) or not math.isfinite(row.pedestal)
                or row.pedestal < 0):
            raise ValueError("invalid background/pedestal in manifest")
        rows.append(row)
    if len(lines) > exposures and any(l.strip() for l in lines[exposures:]):
        raise ValueError("manifest has more rows than expected")
    return rows


@dataclasses.dataclass
class EngineArgs:
    """The 18 positional arguments of ``updc_jwst_c`` (updc_core.c:1566-1572)."""
    manifest: str
    width: int
    height: int
    input_width: int
    input_height: int
    exposures: int
    psf_transposed: int
    iterations: int
    iter_prefix: str
    weight_output: str
    fft_workers: int = 1
    exposure_workers: int = 1
    preprocess_workers: int = 1
    plan_measure: int = 0
    autotune: int = 0
    retune_fft: int = 0
    wisdom_path: str = ""
    save_every: int = 0

    def argv(self) -> List[str]:
        return [str(v) for v in dataclasses.astuple(self)]
