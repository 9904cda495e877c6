"""TEST INFRASTRUCTURE ONLY — ctypes access to the parity oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module.  It loads ``oracle/_build/liboracle.so`` (the C restatement
of the reference solver, see updc_oracle.c) and runs ``oracle/_ref/updc_jwst_c``
(the reference core compiled from its own sources against the FFTW-API shim).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
SHIM_PATH = HERE / "_build" / "libfftw_shim.so"
REF_BINARY = HERE / "_ref" / "updc_jwst_c"
REF_PROJECTOR = HERE / "_ref" / "updc_psf_projector"
# the reference checkout: UPDC_REFERENCE_DIR, by default a sibling of this repository
REFERENCE_SOURCES = Path(os.environ.get("UPDC_REFERENCE_DIR", HERE.parent.parent / "reference")) / "updc" / "c_core"

_lib = None


def build(reference: bool = True) -> None:
    """Compile the oracle (and the reference core when its sources exist)."""
    targets = ["oracle"]
    if reference and (REFERENCE_SOURCES / "updc_core.c").is_file():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.is_file():
            build(reference=False)
        L = ctypes.CDLL(str(LIB_PATH))
        c = ctypes
        L.orc_polygon_area.restype = c.c_float
        L.orc_polygon_area.argtypes = [c.c_void_p, c.c_int]
        L.orc_overlap_area.restype = c.c_float
        L.orc_overlap_area.argtypes = [c.c_void_p, c.c_int, c.c_int]
        L.orc_linkmap_build.argtypes = [c.c_char_p, c.c_int, c.c_int, c.c_int, c.c_int, c.c_char_p,
                                        c.POINTER(c.c_uint64), c.POINTER(c.c_int)]
        L.orc_linkmap_info.argtypes = [c.c_char_p, c.c_int, c.c_int, c.c_int, c.c_int,
                                       c.POINTER(c.c_uint64), c.POINTER(c.c_int)]
        L.orc_linkmap_decode.argtypes = [c.c_char_p, c.c_int, c.c_int, c.c_int, c.c_int,
                                         c.c_void_p, c.c_void_p, c.c_void_p]
        L.orc_next_fast_size.argtypes = [c.c_int]
        L.orc_create.restype = c.c_void_p
        L.orc_create.argtypes = [c.c_int, c.c_char_p] + [c.c_int] * 10 + [c.c_char_p, c.c_int]
        L.orc_iterate.argtypes = [c.c_void_p, c.c_int, c.c_void_p, c.c_void_p, c.c_void_p, c.c_char_p, c.c_int]
        L.orc_plane.restype = c.c_void_p
        L.orc_plane.argtypes = [c.c_void_p, c.c_int]
        L.orc_frozen.restype = c.c_void_p
        L.orc_frozen.argtypes = [c.c_void_p]
        L.orc_scalar.restype = c.c_double
        L.orc_scalar.argtypes = [c.c_void_p, c.c_int]
        L.orc_spectrum.restype = c.c_void_p
        L.orc_spectrum.argtypes = [c.c_void_p, c.c_int]
        L.orc_forward_blur.argtypes = [c.c_void_p, c.c_int]
        L.orc_detector.argtypes = [c.c_void_p, c.c_int, c.c_void_p, c.c_void_p, c.POINTER(c.c_uint64),
                                   c.POINTER(c.c_uint64), c.POINTER(c.c_double), c.c_char_p, c.c_int]
        L.orc_update.argtypes = [c.c_void_p, c.c_char_p, c.c_int]
        L.orc_adjoint.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p]
        L.orc_fft_r2c.argtypes = [c.c_int] * 4 + [c.c_void_p, c.c_void_p]
        L.orc_fft_c2r.argtypes = [c.c_int] * 4 + [c.c_void_p, c.c_void_p]
        _lib = L
    return _lib


# ---------------------------------------------------------------- geometry / LinkMap

def polygon_area(points: np.ndarray) -> float:
    pts = np.ascontiguousarray(points, dtype=np.float64)
    return float(lib().orc_polygon_area(pts.ctypes.data, len(pts)))


def overlap_area(quad: np.ndarray, x: int, y: int) -> float:
    q = np.ascontiguousarray(quad, dtype=np.float64)
    return float(lib().orc_overlap_area(q.ctypes.data, x, y))


def next_fast_size(n: int) -> int:
    return int(lib().orc_next_fast_size(n))


def linkmap_build(vertices: str, iw: int, ih: int, W: int, H: int, out: str):
    nl = ctypes.c_uint64()
    enc = ctypes.c_int()
    rc = lib().orc_linkmap_build(vertices.encode(), iw, ih, W, H, out.encode(), ctypes.byref(nl), ctypes.byref(enc))
    if rc:
        raise RuntimeError("oracle LinkMap build failed")
    return int(nl.value), int(enc.value)


def linkmap_decode(path: str, iw: int, ih: int, W: int, H: int):
    nl = ctypes.c_uint64()
    enc = ctypes.c_int()
    if lib().orc_linkmap_info(path.encode(), iw, ih, W, H, ctypes.byref(nl), ctypes.byref(enc)):
        raise ValueError("invalid or obsolete LinkMap cache")
    n = int(nl.value)
    off = np.zeros(iw * ih + 1, np.uint32)
    tgt = np.zeros(max(n, 1), np.uint32)
    frac = np.zeros(max(n, 1), np.float32)
    if lib().orc_linkmap_decode(path.encode(), iw, ih, W, H, off.ctypes.data, tgt.ctypes.data, frac.ctypes.data):
        raise ValueError("LinkMap decode failed")
    return off, tgt[:n], frac[:n], int(enc.value)


# ---------------------------------------------------------------- solver

class Solver:
    """The oracle solver (FP32 = reference operation order, FP64 = CPU FP64 oracle)."""

    def __init__(self, manifest: str, W: int, H: int, iw: int, ih: int, nexp: int, FW: int, FH: int,
                 precision: int = 32, transposed: int = 0, nthreads: int = 0, reuse_links: bool = True):
        self.W, self.H, self.iw, self.ih, self.nexp, self.FW, self.FH = W, H, iw, ih, nexp, FW, FH
        self.precision = precision
        self.dtype = np.float64 if precision == 64 else np.float32
        nthreads = nthreads or min(8, os.cpu_count() or 1)
        err = ctypes.create_string_buffer(512)
        h = lib().orc_create(precision, str(manifest).encode(), W, H, iw, ih, nexp, transposed, FW, FH,
                             nthreads, 1 if reuse_links else 0, err, 512)
        if not h:
            raise RuntimeError("UPDC_ALL: " + err.value.decode())
        self.h = ctypes.c_void_p(h)
        self.iterations_done = 0

    def _plane(self, which: int, n: int) -> np.ndarray:
        ptr = lib().orc_plane(self.h, which)
        ct = ctypes.c_double if self.precision == 64 else ctypes.c_float
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,))

    @property
    def estimate(self):
        return self._plane(0, self.W * self.H).reshape(self.H, self.W)

    @property
    def coverage(self):
        return self._plane(1, self.W * self.H).reshape(self.H, self.W)

    @property
    def denominator(self):
        return self._plane(2, self.W * self.H).reshape(self.H, self.W)

    @property
    def correction(self):
        return self._plane(3, self.W * self.H).reshape(self.H, self.W)

    @property
    def blur(self):
        return self._plane(4, self.W * self.H).reshape(self.H, self.W)

    @property
    def scatter(self):
        return self._plane(5, self.W * self.H).reshape(self.H, self.W)

    @property
    def sci(self):
        return self._plane(6, self.nexp * self.iw * self.ih).reshape(self.nexp, self.ih, self.iw)

    @property
    def wht(self):
        return self._plane(7, self.nexp * self.iw * self.ih).reshape(self.nexp, self.ih, self.iw)

    @property
    def frozen(self):
        ptr = lib().orc_frozen(self.h)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)),
                                     shape=(self.nexp * self.iw * self.ih,)).reshape(self.nexp, self.ih, self.iw)

    @property
    def weight_scale(self) -> float:
        return lib().orc_scalar(self.h, 0)

    @property
    def max_sensitivity(self) -> float:
        return lib().orc_scalar(self.h, 1)

    def spectrum(self, k: int) -> np.ndarray:
        ptr = lib().orc_spectrum(self.h, k)
        ct = ctypes.c_double if self.precision == 64 else ctypes.c_float
        n = self.FH * (self.FW // 2 + 1) * 2
        a = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,))
        return a.view(np.complex128 if self.precision == 64 else np.complex64).reshape(self.FH, self.FW // 2 + 1)

    def iterate(self, n: int = 1):
        """Run n iterations; returns (new, total, min_raw_mu) arrays of shape (n, nexp)."""
        new = np.zeros((n, self.nexp), np.uint64)
        tot = np.zeros((n, self.nexp), np.uint64)
        mn = np.zeros((n, self.nexp), np.float64)
        err = ctypes.create_string_buffer(512)
        if lib().orc_iterate(self.h, n, new.ctypes.data, tot.ctypes.data, mn.ctypes.data, err, 512):
            raise RuntimeError("UPDC_ALL: " + err.value.decode())
        self.iterations_done += n
        return new, tot, mn

    def forward_blur(self, k: int) -> np.ndarray:
        lib().orc_forward_blur(self.h, k)
        return self.blur.copy()

    def detector(self, k: int, blur: np.ndarray):
        b = np.ascontiguousarray(blur, dtype=self.dtype)
        out = np.zeros_like(b)
        nn, nt, mm = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        if lib().orc_detector(self.h, k, b.ctypes.data, out.ctypes.data, ctypes.byref(nn), ctypes.byref(nt),
                              ctypes.byref(mm), err, 512):
            raise RuntimeError("UPDC_ALL: " + err.value.decode())
        return out, int(nn.value), int(nt.value), float(mm.value)

    def adjoint(self, v: np.ndarray) -> np.ndarray:
        """H^T v for detector planes v (nexp x ih x iw) with the reference's
        scatter and frequency-domain adjoint (updc_core.c:988-995, 1175-1176,
        1280-1287); returns the target plane."""
        a = np.ascontiguousarray(v, dtype=self.dtype)
        out = np.zeros((self.H, self.W), self.dtype)
        lib().orc_adjoint(self.h, a.ctypes.data, out.ctypes.data)
        return out


def fft_r2c(x: np.ndarray, precision: int = 64, nthreads: int = 4) -> np.ndarray:
    dt = np.float64 if precision == 64 else np.float32
    a = np.ascontiguousarray(x, dtype=dt)
    n0, n1 = a.shape
    out = np.zeros((n0, n1 // 2 + 1), np.complex128 if precision == 64 else np.complex64)
    lib().orc_fft_r2c(precision, n0, n1, nthreads, a.ctypes.data, out.ctypes.data)
    return out


# ---------------------------------------------------------------- the compiled reference

def run_reference(args: Sequence[str], env: Optional[dict] = None, timeout: float = 3600.0):
    """Run the reference core (oracle/_ref/updc_jwst_c) with the 18-argument contract."""
    if not REF_BINARY.is_file():
        raise FileNotFoundError(f"reference core not built: {REF_BINARY}")
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([str(REF_BINARY), *map(str, args)], capture_output=True, text=True,
                          env=e, timeout=timeout)
