"""Batched cutout fields through the C ABI (updc_batch_*).

    b = Batch(form="fp32", autotune=True)
    for ds in datasets:
        b.add_field(ds.manifest, W, H, iw, ih, nexp)
    b.setup()
    recs = b.iterate(30)            # one graph of 30 iterations over every field
    x = b.field(3).plane("estimate")

Each field is solved exactly as its own ``Engine`` would solve it
(updc/c_core/updc_core.c:1410-1456 per field); the batch only changes how
the work is launched: one persistent launch per stage over all fields.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import check
from .engine import Engine


class _FieldView(Engine):
    """Plane and scalar access to one field of a batch (owned by the batch)."""

    def __init__(self, handle, L, form, W, H, iw, ih, nexp):
        self._h = handle
        self._L = L
        self.form = form
        self.dtype = np.float64 if form == "fp64" else np.float32
        self.W, self.H, self.iw, self.ih, self.nexp = W, H, iw, ih, nexp
        self.iterations_done = 0

    def close(self) -> None:       # the batch owns the field
        self._h = None


class Batch:
    def __init__(self, form: str = "fp32", device: int = 0, autotune: bool = False,
                 tune_cache_dir: Optional[str] = None, reuse_links: bool = True):
        L = _lib.load()
        opt = _lib.Options()
        L.updc_default_options(ctypes.byref(opt))
        opt.form = _lib.FORMS[form]
        opt.device = device
        opt.reuse_links = 1 if reuse_links else 0
        opt.autotune = 1 if autotune else 0
        self._cache_dir = str(tune_cache_dir).encode() if tune_cache_dir else None
        opt.tune_cache_dir = self._cache_dir
        h = ctypes.c_void_p()
        check(L.updc_batch_create(ctypes.byref(opt), ctypes.byref(h)))
        self._h, self._L, self.form = h, L, form
        self._shapes = []

    def close(self) -> None:
        if self._h:
            self._L.updc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_field(self, manifest, width: int, height: int, input_width: int, input_height: int,
                  exposures: int, psf_transposed: int = 0) -> int:
        check(self._L.updc_batch_add_field(self._h, str(manifest).encode(), width, height, input_width,
                                           input_height, exposures, psf_transposed))
        self._shapes.append((width, height, input_width, input_height, exposures))
        return len(self._shapes) - 1

    def setup(self) -> "Batch":
        check(self._L.updc_batch_setup(self._h))
        return self

    @property
    def fields(self) -> int:
        return len(self._shapes)

    def units(self, stage: int) -> int:
        return int(self._L.updc_batch_units(self._h, stage))

    def field(self, i: int) -> Engine:
        fh = self._L.updc_batch_field(self._h, i)
        if not fh:
            raise IndexError(i)
        W, H, iw, ih, nexp = self._shapes[i]
        return _FieldView(ctypes.c_void_p(fh), self._L, self.form, W, H, iw, ih, nexp)

    def iterate(self, n: int = 1, check_each: bool = False) -> List[dict]:
        nf = self.fields
        ne = sum(s[4] for s in self._shapes)
        sec = np.zeros(n, np.float64)
        ssum = np.zeros((n, nf), np.float64)
        neg = np.zeros((n, nf), np.uint64)
        frz = np.zeros((n, ne), np.uint64)
        check(self._L.updc_batch_iterate(self._h, n, 1 if check_each else 0, sec.ctypes.data, ssum.ctypes.data,
                                         neg.ctypes.data, frz.ctypes.data))
        return [{"seconds": float(sec[i]), "signed_sum": ssum[i], "negative": neg[i], "total_frozen": frz[i]}
                for i in range(n)]
