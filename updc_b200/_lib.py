"""ctypes binding of libupdc_b200.so (include/updc_b200.h).

The library is built in-tree by ``python -m updc_b200.build``.  Loading fails
loudly when it is missing: there is no CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path
from typing import List

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libupdc_b200.so"
EXE_PATH = PKG / "bin" / "updc_jwst_c"
HEADER = PKG.parent / "include" / "updc_b200.h"

FORM_FP32, FORM_FP64, FORM_FP32_KAHAN, FORM_FP32_REFERENCE = 0, 1, 2, 3
FORMS = {"fp32": FORM_FP32, "fp64": FORM_FP64, "fp32-kahan": FORM_FP32_KAHAN,
         "fp32-reference": FORM_FP32_REFERENCE}

(PLANE_ESTIMATE, PLANE_COVERAGE, PLANE_DENOMINATOR, PLANE_CORRECTION, PLANE_BLUR, PLANE_SCATTER,
 PLANE_SCIENCE, PLANE_WEIGHT, PLANE_WR, PLANE_FROZEN) = range(10)


class Options(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int), ("compensated_mu", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("device", ctypes.c_int), ("reuse_links", ctypes.c_int), ("verbose", ctypes.c_int),
                ("fft_width", ctypes.c_int), ("fft_height", ctypes.c_int), ("stage_timing", ctypes.c_int),
                ("autotune", ctypes.c_int), ("retune", ctypes.c_int), ("tune_cache_dir", ctypes.c_char_p),
                ("fft_linear", ctypes.c_int)]


class IterStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("signed_sum", ctypes.c_double), ("negative", ctypes.c_uint64),
                ("stage_seconds", ctypes.c_double * 8)]


class PreprocessMetrics(ctypes.Structure):
    _fields_ = [(name, ctypes.c_double) for name in (
        "background", "background_sigma", "poisson_pedestal", "auto_positivity_pedestal", "requested_pedestal",
        "min_valid_science", "sky_var_poisson", "wht_valid_median")] + \
        [(name, ctypes.c_int64) for name in ("base_invalid", "nonpositive_valid_before_pedestal",
                                             "nonpositive_after_pedestal", "wht_zero")] + \
        [("clip_passes", ctypes.c_int32), ("std_fallbacks", ctypes.c_int32)]


class UpdcError(RuntimeError):
    """A failure reported by the engine; str() is the reference core's message."""


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.is_file():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m updc_b200.build` "
                          "(the solver has no CPU fallback)")
    L = ctypes.CDLL(str(LIB_PATH))
    c = ctypes
    P = c.c_void_p
    L.updc_version.restype = c.c_char_p
    L.updc_last_error.restype = c.c_char_p
    L.updc_default_options.argtypes = [c.POINTER(Options)]
    L.updc_create.argtypes = [c.POINTER(Options), c.POINTER(P)]
    L.updc_destroy.argtypes = [P]
    L.updc_load_manifest.argtypes = [P, c.c_char_p] + [c.c_int] * 6
    L.updc_setup.argtypes = [P]
    L.updc_iterate.argtypes = [P, c.c_int, c.c_int, c.POINTER(IterStats), P, P, P]
    L.updc_read_plane.argtypes = [P, c.c_int, c.c_int, P, c.c_int]
    L.updc_write_plane.argtypes = [P, c.c_int, c.c_int, P, c.c_int]
    L.updc_scalar.restype = c.c_double
    L.updc_scalar.argtypes = [P, c.c_int]
    L.updc_device_bytes.restype = c.c_size_t
    L.updc_device_bytes.argtypes = [P]
    L.updc_set_stage_timing.argtypes = [P, c.c_int]
    L.updc_fft_radices.argtypes = [P, c.c_int, P, c.c_int, c.POINTER(c.c_int)]
    L.updc_stage_forward.argtypes = [P]
    L.updc_stage_detector.argtypes = [P, P, P, P]
    L.updc_stage_correction.argtypes = [P]
    L.updc_stage_update.argtypes = [P, c.POINTER(c.c_double), c.POINTER(c.c_uint64)]
    L.updc_update_noalloc.argtypes = [P, P, P, c.c_uint64, c.c_float, P, c.POINTER(c.c_double), c.POINTER(c.c_uint64)]
    L.updc_set_exposure_offsets.argtypes = [P, c.c_int, c.c_double, c.c_double]
    L.updc_set_psf.argtypes = [P, c.c_int, P, c.c_int, c.c_int, c.c_int]
    L.updc_nll.argtypes = [P, P]
    L.updc_nll_partials.argtypes = [P, P, c.c_size_t, c.POINTER(c.c_size_t)]
    L.updc_nll_adjoint.argtypes = [P]
    L.updc_psf_gradient.argtypes = [P, c.c_int, P]
    L.updc_copy_plane_device.argtypes = [P, c.c_int, c.c_int, P, c.c_int, c.c_int, P]
    L.updc_batch_create.argtypes = [c.POINTER(Options), c.POINTER(P)]
    L.updc_batch_destroy.argtypes = [P]
    L.updc_batch_add_field.argtypes = [P, c.c_char_p] + [c.c_int] * 6
    L.updc_batch_setup.argtypes = [P]
    L.updc_batch_fields.argtypes = [P]
    L.updc_batch_field.restype = P
    L.updc_batch_field.argtypes = [P, c.c_int]
    L.updc_batch_units.restype = c.c_size_t
    L.updc_batch_units.argtypes = [P, c.c_int]
    L.updc_batch_iterate.argtypes = [P, c.c_int, c.c_int, P, P, P, P]
    L.updc_set_active_exposures.argtypes = [P, c.c_int, c.c_int]
    L.updc_refresh_sensitivity.argtypes = [P]
    L.updc_device_wait_check.argtypes = [c.c_uint32]
    L.updc_finish_shard_setup.argtypes = [P]
    L.updc_plane_device_pointer.argtypes = [P, c.c_int, c.POINTER(c.c_void_p)]
    L.updc_engine_stream.argtypes = [P, c.POINTER(c.c_void_p)]
    L.updc_enqueue_partial.argtypes = [P]
    L.updc_enqueue_update.argtypes = [P]
    L.updc_finish_iteration.argtypes = [P, c.POINTER(c.c_double), c.POINTER(c.c_uint64), P, P, P]
    L.updc_save_state.argtypes = [P, c.c_char_p, c.c_uint64]
    L.updc_load_state.argtypes = [P, c.c_char_p, c.POINTER(c.c_uint64)]
    L.updc_link_count.restype = c.c_uint64
    L.updc_link_count.argtypes = [P, c.c_int]
    L.updc_link_encoding.argtypes = [P, c.c_int]
    L.updc_decode_links.argtypes = [P, c.c_int, P]
    L.updc_build_linkmap.argtypes = [c.c_char_p, c.c_char_p] + [c.c_int] * 4 + [c.POINTER(c.c_uint64), c.POINTER(c.c_int)]
    L.updc_preprocess_exposure.argtypes = [P, P, P, P, P, c.c_int64, c.c_int, c.c_uint32, c.c_double, c.c_char_p,
                                           P, P, c.POINTER(PreprocessMetrics), c.c_int, P]
    L.updc_robust_background.argtypes = [P, P, c.c_int64, c.c_int, P, c.POINTER(c.c_double),
                                         c.POINTER(c.c_double), c.POINTER(c.c_int), c.c_int, P]
    L.updc_polygon_area.restype = c.c_float
    L.updc_polygon_area.argtypes = [P, c.c_int]
    L.updc_overlap_area.restype = c.c_float
    L.updc_overlap_area.argtypes = [P, c.c_int, c.c_int]
    L.updc_self_test.argtypes = [c.c_char_p, c.c_size_t]
    L.updc_all.argtypes = [c.c_char_p] + [c.c_int] * 7 + [c.c_char_p, c.c_char_p] + [c.c_int] * 6 + [c.c_char_p, c.c_int]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc:
        raise UpdcError(load().updc_last_error().decode())


def declared_functions() -> List[str]:
    """Names of the functions declared in include/updc_b200.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(updc_\w+|UPDC_ALL)\s*\(", text)
    return sorted(set(names))
