"""Python host API of the B200 UPDC engine.

``Engine`` mirrors the stages of the reference core's UPDC_ALL
(updc/c_core/updc_core.c:1289-1543) behind the engine handoff's inputs:

    eng = Engine(form="fp32")
    eng.load(manifest, W, H, iw, ih, nexp)     # parse_manifest, core:426-461
    eng.setup()                                 # core:1330-1398
    stats = eng.iterate(39)                     # core:1410-1479
    x = eng.plane("estimate")

``run_engine_args`` is the 18-argument call (the argv contract of
``updc_jwst_c``, core:1566-1572) without a process boundary; the executable
``updc_b200/bin/updc_jwst_c`` is the drop-in for ``build.c_core_binary``.
Failures raise ``UpdcError`` with the reference's message.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import UpdcError, check

PLANES = {"estimate": _lib.PLANE_ESTIMATE, "coverage": _lib.PLANE_COVERAGE,
          "denominator": _lib.PLANE_DENOMINATOR, "correction": _lib.PLANE_CORRECTION,
          "blur": _lib.PLANE_BLUR, "scatter": _lib.PLANE_SCATTER, "science": _lib.PLANE_SCIENCE,
          "weight": _lib.PLANE_WEIGHT, "wr": _lib.PLANE_WR, "frozen": _lib.PLANE_FROZEN}
TARGET_PLANES = {"estimate", "coverage", "denominator", "correction", "blur", "scatter"}


@dataclasses.dataclass
class IterationStats:
    seconds: float
    signed_sum: float
    negative: int
    new_frozen: np.ndarray     # per exposure
    total_frozen: np.ndarray
    min_raw_mu: np.ndarray
    stage_seconds: np.ndarray


class Engine:
    """One solver instance on one GPU (the handle of include/updc_b200.h)."""

    def __init__(self, form: str = "fp32", device: int = 0, use_graph: bool = True,
                 reuse_links: bool = True, compensated_mu: Optional[bool] = None, verbose: bool = False,
                 fft_shape: Optional[tuple] = None, stage_timing: bool = False, autotune: bool = False,
                 retune: bool = False, tune_cache_dir: Optional[str] = None, fft_linear: bool = False):
        L = _lib.load()
        opt = _lib.Options()
        L.updc_default_options(ctypes.byref(opt))
        opt.form = _lib.FORMS[form]
        opt.device = device
        opt.use_graph = 1 if use_graph else 0
        opt.reuse_links = 1 if reuse_links else 0
        opt.compensated_mu = -1 if compensated_mu is None else int(bool(compensated_mu))
        opt.verbose = 1 if verbose else 0
        opt.stage_timing = 1 if stage_timing else 0
        opt.autotune = 1 if autotune else 0
        opt.retune = 1 if retune else 0
        self._cache_dir = str(tune_cache_dir).encode() if tune_cache_dir else None
        opt.tune_cache_dir = self._cache_dir
        opt.fft_linear = 1 if fft_linear else 0
        if fft_shape:
            opt.fft_width, opt.fft_height = fft_shape
        h = ctypes.c_void_p()
        check(L.updc_create(ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self._L = L
        self.form = form
        self.dtype = np.float64 if form == "fp64" else np.float32
        self.W = self.H = self.iw = self.ih = self.nexp = 0
        self.iterations_done = 0

    def close(self) -> None:
        if self._h:
            self._L.updc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ stages
    def load(self, manifest: str, width: int, height: int, input_width: int, input_height: int,
             exposures: int, psf_transposed: int = 0) -> "Engine":
        check(self._L.updc_load_manifest(self._h, str(manifest).encode(), width, height, input_width,
                                         input_height, exposures, psf_transposed))
        self.W, self.H, self.iw, self.ih, self.nexp = width, height, input_width, input_height, exposures
        return self

    def setup(self) -> "Engine":
        check(self._L.updc_setup(self._h))
        return self

    def iterate(self, n: int = 1, check_each: bool = True) -> List[IterationStats]:
        st = (_lib.IterStats * max(n, 1))()
        new = np.zeros((n, self.nexp), np.uint64)
        tot = np.zeros((n, self.nexp), np.uint64)
        mn = np.zeros((n, self.nexp), np.float64)
        check(self._L.updc_iterate(self._h, n, 1 if check_each else 0, st, new.ctypes.data,
                                   tot.ctypes.data, mn.ctypes.data))
        self.iterations_done += n
        return [IterationStats(st[i].seconds, st[i].signed_sum, int(st[i].negative), new[i], tot[i], mn[i],
                               np.array(st[i].stage_seconds[:])) for i in range(n)]

    # ------------------------------------------------------------------ data access
    def plane(self, name: str, exposure: int = 0, as_double: bool = False) -> np.ndarray:
        which = PLANES[name]
        if name == "frozen":
            out = np.zeros((self.ih, self.iw), np.uint8)
            check(self._L.updc_read_plane(self._h, which, exposure, out.ctypes.data, 0))
            return out
        shape = (self.H, self.W) if name in TARGET_PLANES else (self.ih, self.iw)
        out = np.zeros(shape, np.float64 if as_double else np.float32)
        check(self._L.updc_read_plane(self._h, which, exposure, out.ctypes.data, 1 if as_double else 0))
        return out

    def set_plane(self, name: str, data: np.ndarray, exposure: int = 0) -> None:
        """Write a plane from a float32 or float64 array (no host-side copy when
        the array is already contiguous; pinned arrays copy at full bandwidth)."""
        which = PLANES[name]
        if name == "frozen":
            a = np.ascontiguousarray(data, np.uint8)
            check(self._L.updc_write_plane(self._h, which, exposure, a.ctypes.data, 0))
            return
        if data.dtype not in (np.float32, np.float64):
            data = data.astype(np.float64)
        a = np.ascontiguousarray(data)
        check(self._L.updc_write_plane(self._h, which, exposure, a.ctypes.data, 1 if a.dtype == np.float64 else 0))

    def read_plane_into(self, name: str, out: np.ndarray, exposure: int = 0) -> np.ndarray:
        """Copy a plane into a caller-owned contiguous float32/float64 array."""
        if not out.flags.c_contiguous or out.dtype not in (np.float32, np.float64):
            raise ValueError("out must be a contiguous float32 or float64 array")
        check(self._L.updc_read_plane(self._h, PLANES[name], exposure, out.ctypes.data,
                                      1 if out.dtype == np.float64 else 0))
        return out

    def set_stage_timing(self, on: bool) -> None:
        check(self._L.updc_set_stage_timing(self._h, 1 if on else 0))

    def scalar(self, which: int) -> float:
        return float(self._L.updc_scalar(self._h, which))

    @property
    def weight_scale(self) -> float:
        return self.scalar(0)

    @property
    def max_sensitivity(self) -> float:
        return self.scalar(1)

    @property
    def fft_shape(self) -> tuple:
        return int(self.scalar(2)), int(self.scalar(3))

    def fft_radices(self, axis: int) -> List[int]:
        """Radix split of the row (axis 0, FW/2 points) or column (axis 1, FH points) transform."""
        buf = (ctypes.c_int * 32)()
        n = ctypes.c_int()
        check(self._L.updc_fft_radices(self._h, axis, buf, 32, ctypes.byref(n)))
        return list(buf[:n.value])

    @property
    def autotune_info(self) -> dict:
        return {"seconds": self.scalar(7), "plans_timed": int(self.scalar(8)), "cache_hit": bool(self.scalar(9)),
                "modelled_ms": self.scalar(10)}

    @property
    def kernel_variants(self) -> dict:
        """Which specialised kernels the iteration runs: row / column transforms
        compiled for their radix sequence, the adjoint gather fused into the
        scatter row transform (no scatter plane), four-step rows and columns
        for FFT shapes beyond one block, and two-row tiles of 1024 threads for
        FP32 rows of more than half a block."""
        v = int(self.scalar(11))
        return {"compiled_rows": bool(v & 1), "compiled_columns": bool(v & 2), "fused_gather": bool(v & 4),
                "long_rows": bool(v & 8), "long_columns": bool(v & 16), "wide_rows": bool(v & 32)}

    @property
    def masked_pixels(self) -> int:
        return int(self.scalar(4))

    @property
    def device_bytes(self) -> int:
        return int(self._L.updc_device_bytes(self._h))

    # ------------------------------------------------------------------ stage hooks
    def stage_forward(self) -> None:
        check(self._L.updc_stage_forward(self._h))

    def stage_detector(self):
        new = np.zeros(self.nexp, np.uint64)
        tot = np.zeros(self.nexp, np.uint64)
        mn = np.zeros(self.nexp, np.float64)
        check(self._L.updc_stage_detector(self._h, new.ctypes.data, tot.ctypes.data, mn.ctypes.data))
        return new, tot, mn

    def stage_correction(self) -> None:
        check(self._L.updc_stage_correction(self._h))

    def stage_update(self):
        s = ctypes.c_double()
        n = ctypes.c_uint64()
        check(self._L.updc_stage_update(self._h, ctypes.byref(s), ctypes.byref(n)))
        return s.value, int(n.value)

    # ------------------------------------------------------------------ checkpoint / resume
    def save_state(self, path, iteration: Optional[int] = None) -> None:
        """Write the estimate and the FreezeMu masks (with the iteration count)."""
        check(self._L.updc_save_state(self._h, str(path).encode(),
                                      self.iterations_done if iteration is None else iteration))

    def load_state(self, path) -> int:
        """Restore a state written by save_state on the same field and form;
        returns its iteration count (also set as iterations_done)."""
        it = ctypes.c_uint64()
        check(self._L.updc_load_state(self._h, str(path).encode(), ctypes.byref(it)))
        self.iterations_done = int(it.value)
        return self.iterations_done

    # ------------------------------------------------------------------ exposure shards
    def set_active_exposures(self, first: int, count: int) -> None:
        check(self._L.updc_set_active_exposures(self._h, first, count))

    def refresh_sensitivity(self) -> None:
        check(self._L.updc_refresh_sensitivity(self._h))

    def finish_shard_setup(self) -> None:
        """After a shard setup (set_active_exposures before setup) and the sum
        of its partial planes over the shards: the drizzle estimate and the
        maximum sensitivity."""
        check(self._L.updc_finish_shard_setup(self._h))

    def plane_device_pointer(self, name: str) -> int:
        """The engine's own device address of a target plane (W x H elements
        of the form's precision), valid until close()."""
        p = ctypes.c_void_p()
        check(self._L.updc_plane_device_pointer(self._h, PLANES[name], ctypes.byref(p)))
        return int(p.value or 0)

    def stream_handle(self) -> int:
        """The cudaStream_t every launch of the engine is issued on."""
        p = ctypes.c_void_p()
        check(self._L.updc_engine_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def enqueue_partial(self) -> None:
        """Partial correction of the active exposures into the correction
        plane, enqueued on the engine's stream without waiting."""
        check(self._L.updc_enqueue_partial(self._h))

    def enqueue_update(self) -> None:
        """The update from the correction plane as it stands, enqueued on the
        engine's stream without waiting."""
        check(self._L.updc_enqueue_update(self._h))

    def finish_iteration(self):
        """Waits for the engine's stream; returns (signed_sum, negative,
        new_frozen, total_frozen, min_raw_mu) of the iteration just enqueued."""
        s = ctypes.c_double()
        n = ctypes.c_uint64()
        new = np.zeros(self.nexp, np.uint64)
        tot = np.zeros(self.nexp, np.uint64)
        mn = np.zeros(self.nexp, np.float64)
        check(self._L.updc_finish_iteration(self._h, ctypes.byref(s), ctypes.byref(n), new.ctypes.data,
                                            tot.ctypes.data, mn.ctypes.data))
        self.iterations_done += 1
        return float(s.value), int(n.value), new, tot, mn

    # ------------------------------------------------------------------ differentiable model
    def set_exposure_offsets(self, exposure: int, background: float, pedestal: float) -> None:
        check(self._L.updc_set_exposure_offsets(self._h, exposure, float(background), float(pedestal)))

    def set_psf(self, exposure: int, psf: np.ndarray) -> None:
        """Replace an exposure's PSF (2-D float32 or float64 array, manifest layout)."""
        a = np.ascontiguousarray(psf, np.float64 if psf.dtype == np.float64 else np.float32)
        check(self._L.updc_set_psf(self._h, exposure, a.ctypes.data, a.shape[1], a.shape[0],
                                   1 if a.dtype == np.float64 else 0))

    def nll(self) -> np.ndarray:
        """Forward model of the current estimate; per exposure
        [L_k, sum r, sum W log mu, pixels left out] (see updc_nll)."""
        out = np.zeros((self.nexp, 4), np.float64)
        check(self._L.updc_nll(self._h, out.ctypes.data))
        return out

    def nll_partials(self) -> np.ndarray:
        """Per-block partial sums behind the last nll(): (exposures, blocks, 4)."""
        n = ctypes.c_size_t()
        check(self._L.updc_nll_partials(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.float64)
        check(self._L.updc_nll_partials(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out.reshape(self.nexp, -1, 4)

    def nll_adjoint(self) -> None:
        check(self._L.updc_nll_adjoint(self._h))

    def psf_gradient(self, exposure: int, shape: tuple) -> np.ndarray:
        out = np.zeros(shape, np.float64)
        check(self._L.updc_psf_gradient(self._h, exposure, out.ctypes.data))
        return out

    def copy_plane_device(self, name: str, ptr: int, to_engine: bool, as_double: bool, exposure: int = 0,
                          stream: int = 0) -> None:
        check(self._L.updc_copy_plane_device(self._h, PLANES[name], exposure, ptr, 1 if to_engine else 0,
                                             1 if as_double else 0, stream or None))

    # ------------------------------------------------------------------ LinkMaps
    def link_count(self, exposure: int) -> int:
        return int(self._L.updc_link_count(self._h, exposure))

    def link_encoding(self, exposure: int) -> int:
        return int(self._L.updc_link_encoding(self._h, exposure))

    def decode_links(self, exposure: int) -> np.ndarray:
        out = np.zeros(max(self.link_count(exposure), 1), np.uint32)
        check(self._L.updc_decode_links(self._h, exposure, out.ctypes.data))
        return out[:self.link_count(exposure)]


def build_linkmap(vertices: str, links: str, input_width: int, input_height: int, width: int, height: int):
    """Build a LinkMap v2 file on the GPU; returns (nlinks, encoding)."""
    L = _lib.load()
    nl = ctypes.c_uint64()
    enc = ctypes.c_int()
    check(L.updc_build_linkmap(str(vertices).encode(), str(links).encode(), input_width, input_height, width,
                               height, ctypes.byref(nl), ctypes.byref(enc)))
    return int(nl.value), int(enc.value)


def update_noalloc(correction: int, denominator: int, estimate: int, n: int, max_sensitivity: float,
                   stream: int = 0):
    """x *= C/D on caller-owned FP32 device planes (addresses as ints) with no
    device allocation; returns (signed_sum, negative).  Calls that overlap in
    time on one device race on the shared scratch."""
    s = ctypes.c_double()
    neg = ctypes.c_uint64()
    check(_lib.load().updc_update_noalloc(correction, denominator, estimate, n, max_sensitivity, stream or None,
                                          ctypes.byref(s), ctypes.byref(neg)))
    return float(s.value), int(neg.value)


def polygon_area(points: np.ndarray) -> float:
    p = np.ascontiguousarray(points, np.float64)
    return float(_lib.load().updc_polygon_area(p.ctypes.data, len(p)))


def overlap_area(quad: np.ndarray, x: int, y: int) -> float:
    q = np.ascontiguousarray(quad, np.float64)
    return float(_lib.load().updc_overlap_area(q.ctypes.data, x, y))


def self_test() -> str:
    buf = ctypes.create_string_buffer(256)
    rc = _lib.load().updc_self_test(buf, 256)
    if rc:
        raise UpdcError(buf.value.decode())
    return buf.value.decode()


def run_engine_args(args) -> None:
    """The 18-argument solve (updc_core.c:1289-1293) in-process; raises UpdcError."""
    a = [str(v) for v in (args.argv() if hasattr(args, "argv") else args)]
    if len(a) != 18:
        raise ValueError("the engine handoff has 18 arguments")
    L = _lib.load()
    ints = [int(v) for v in a[1:8]] + [int(v) for v in a[10:16]]
    check(L.updc_all(a[0].encode(), *ints[:7], a[8].encode(), a[9].encode(), *ints[7:13], a[16].encode(),
                     int(a[17])))
