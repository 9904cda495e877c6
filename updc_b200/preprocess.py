"""Per-exposure weight preprocessing on the GPU, behind the reference's own
function names (updc/_engine.py:287-408).

``prepare_weighted_inputs`` turns each Level-2 exposure (SCI, DQ,
VAR_POISSON, VAR_RNOISE, VAR_FLAT) into the raw float32 SCI and WHT planes of
the engine handoff and the per-exposure metrics record, printing the same log
line, writing the same files and raising the same ValueErrors as the
reference.  The numeric work — base-valid mask, asymmetric sigma clipping of
the sky, sky VAR_POISSON median, weights, pedestals, WHT — runs in
``libupdc_b200.so`` (``updc_preprocess_exposure``) with results identical to
the reference's NumPy code; there is no CPU path.

Reading FITS is the caller's: the reference opens the files with astropy.
``read_planes`` (a callable path -> mapping of the five plane names to arrays)
replaces that step; the default reads ``.npz`` files and, where astropy is
installed, FITS files.
"""
from __future__ import annotations

import ctypes
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path
from typing import Callable, Mapping, Optional, Sequence

import numpy as np

from . import _lib

PLANES = ("SCI", "DQ", "VAR_POISSON", "VAR_RNOISE", "VAR_FLAT")
WEIGHT_MODES = {"mask": 0, "rnoise-sky": 1, "totalvar": 2}
STATUS_UNKNOWN_MODE = 3


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _raise(rc: int, mode: str) -> None:
    if rc == 0:
        return
    msg = _lib.load().updc_last_error().decode()
    if rc == STATUS_UNKNOWN_MODE:
        raise ValueError(mode)
    if rc == 1:
        raise ValueError(msg)
    raise _lib.UpdcError(msg)


def robust_background_mask(science, base_valid, max_iter: int = 6):
    """Asymmetric sigma clipping of SCI over ``base_valid`` (_engine.py:287-310):
    returns (mask, background, sigma) as the reference does."""
    L = _lib.load()
    sci = np.ascontiguousarray(science, dtype=np.float32)
    valid = np.ascontiguousarray(base_valid, dtype=np.bool_)
    if valid.shape != sci.shape:
        raise ValueError("base_valid and science differ in shape")
    mask = np.empty(sci.shape, dtype=np.bool_)
    bg, sig, passes = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = L.updc_robust_background(_ptr(sci), _ptr(valid), sci.size, int(max_iter), _ptr(mask), ctypes.byref(bg),
                                  ctypes.byref(sig), ctypes.byref(passes), 0, None)
    _raise(rc, "")
    return mask, bg.value, sig.value


def _is_cuda_tensor(a) -> bool:
    return getattr(a, "is_cuda", False)


def prepare_exposure(science, dq, var_poisson, var_rnoise, var_flat, weight_mode: str, bad_dq_mask: int,
                     pedestal_sigma: float, source: str = "", sky_mask: bool = False):
    """The numeric steps of prepare_one (_engine.py:356-397) for one exposure.

    Inputs are NumPy arrays (host; copied to the GPU and back) or CUDA torch
    tensors of the same dtypes (float32 SCI, uint32/int32 DQ, float64
    variances), used in place on torch's current stream.  Returns
    ``(wht, metrics, sky)``: the float32 WHT plane (the input's kind), the
    metric fields of the reference's record (without "exposure"/"source";
    plus "clip_passes" and "std_fallbacks") and the final sky mask (or None).
    """
    L = _lib.load()
    code = WEIGHT_MODES.get(weight_mode, -1)
    m = _lib.PreprocessMetrics()
    if all(_is_cuda_tensor(a) for a in (science, dq, var_poisson, var_rnoise, var_flat)):
        import torch
        planes = [science.contiguous(), dq.contiguous(), var_poisson.contiguous(), var_rnoise.contiguous(),
                  var_flat.contiguous()]
        want = (torch.float32, (torch.int32, torch.uint32), torch.float64, torch.float64, torch.float64)
        for t, dt in zip(planes, want):
            if t.dtype not in (dt if isinstance(dt, tuple) else (dt,)):
                raise TypeError(f"plane dtype {t.dtype}, expected {dt}")
        if len({t.numel() for t in planes}) != 1:
            raise ValueError("Variance/DQ shape mismatch")
        wht = torch.empty(science.shape, dtype=torch.float32, device=science.device)
        sky = torch.empty(science.shape, dtype=torch.uint8, device=science.device) if sky_mask else None
        stream = torch.cuda.current_stream(science.device).cuda_stream
        with torch.cuda.device(science.device):
            rc = L.updc_preprocess_exposure(*[ctypes.c_void_p(t.data_ptr()) for t in planes], science.numel(), code,
                                            int(bad_dq_mask) & 0xFFFFFFFF, float(pedestal_sigma),
                                            str(source).encode(), ctypes.c_void_p(wht.data_ptr()),
                                            ctypes.c_void_p(sky.data_ptr()) if sky is not None else None,
                                            ctypes.byref(m), 1, ctypes.c_void_p(stream))
        sky = sky.bool() if sky is not None else None
    else:
        sci = np.ascontiguousarray(science, dtype=np.float32)
        planes = [sci, np.ascontiguousarray(dq, dtype=np.uint32)] + \
            [np.ascontiguousarray(v, dtype=np.float64) for v in (var_poisson, var_rnoise, var_flat)]
        if any(a.shape != sci.shape for a in planes):
            raise ValueError("Variance/DQ shape mismatch")
        wht = np.empty(sci.shape, dtype=np.float32)
        sky = np.empty(sci.shape, dtype=np.bool_) if sky_mask else None
        rc = L.updc_preprocess_exposure(*[_ptr(a) for a in planes], sci.size, code, int(bad_dq_mask) & 0xFFFFFFFF,
                                        float(pedestal_sigma), str(source).encode(), _ptr(wht),
                                        _ptr(sky) if sky is not None else None, ctypes.byref(m), 0, None)
    _raise(rc, weight_mode)
    metrics = {
        "background": m.background, "background_sigma": m.background_sigma, "poisson_pedestal": m.poisson_pedestal,
        "auto_positivity_pedestal": m.auto_positivity_pedestal, "requested_pedestal": m.requested_pedestal,
        "min_valid_science": m.min_valid_science, "sky_var_poisson": m.sky_var_poisson, "weight_mode": weight_mode,
        "base_invalid": m.base_invalid, "nonpositive_valid_before_pedestal": m.nonpositive_valid_before_pedestal,
        "nonpositive_after_pedestal": m.nonpositive_after_pedestal, "wht_zero": m.wht_zero,
        "wht_valid_median": m.wht_valid_median, "clip_passes": m.clip_passes, "std_fallbacks": m.std_fallbacks,
    }
    return wht, metrics, sky


def default_read_planes(path: Path) -> Mapping[str, np.ndarray]:
    """The five Level-2 planes of one exposure: from an .npz file, or from a
    FITS file through astropy (the reference's reader) where it is installed."""
    path = Path(path)
    if path.suffix == ".npz":
        with np.load(path) as z:
            return {k: z[k] for k in z.files}
    try:
        from astropy.io import fits
    except ImportError as exc:
        raise ImportError(f"reading {path} needs astropy; pass read_planes= to supply the planes") from exc
    with fits.open(path, memmap=False) as h:
        return {name: h[name].data for name in PLANES if name in h}


def prepare_weighted_inputs(images: Sequence[Path], directory: Path, weight_mode: str, bad_dq_mask: int,
                            pedestal_sigma: float, input_shape, preprocess_workers: int = 1,
                            read_planes: Optional[Callable[[Path], Mapping[str, np.ndarray]]] = None):
    """Raw float32 SCI/WHT working planes for the engine (_engine.py:336-408):
    returns ``(prepared, metrics)`` — [(science_raw, weight_raw)] and the
    metric records — and prints one log line per exposure, in exposure order."""
    read = read_planes or default_read_planes
    directory = Path(directory)
    input_shape = tuple(input_shape)

    def prepare_one(item):
        index, path = item
        h = read(path)
        for name in PLANES:
            if name not in h:
                raise ValueError(f"Missing {name} in {path}")
        science = np.asarray(h["SCI"], dtype=np.float32)
        dq = np.asarray(h["DQ"], dtype=np.uint32)
        var_p, var_r, var_f = (np.asarray(h[k], dtype=np.float64) for k in ("VAR_POISSON", "VAR_RNOISE", "VAR_FLAT"))
        if science.shape != input_shape:
            raise ValueError(f"Unexpected SCI shape {science.shape} in {path}")
        if any(a.shape != science.shape for a in (dq, var_p, var_r, var_f)):
            raise ValueError(f"Variance/DQ shape mismatch in {path}")
        wht, m, _ = prepare_exposure(science, dq, var_p, var_r, var_f, weight_mode, bad_dq_mask, pedestal_sigma,
                                     str(path))
        science_raw = directory / f"level2_science_{index:03d}.f32"
        weight_raw = directory / f"level2_weight_{index:03d}.f32"
        np.asarray(science, dtype="<f4").tofile(science_raw)
        np.asarray(wht, dtype="<f4").tofile(weight_raw)
        metric = {"exposure": index, "source": str(path)}
        metric.update({k: v for k, v in m.items() if k not in ("clip_passes", "std_fallbacks")})
        log = (f"Input {index}/{len(images)}: B={m['background']:.8g}, sigma={m['background_sigma']:.8g}, "
               f"pedestal={m['poisson_pedestal']:.8g} (auto={m['auto_positivity_pedestal']:.8g}), "
               f"SCI<=0 retained={m['nonpositive_valid_before_pedestal']}, zero-WHT={m['wht_zero']}")
        return (science_raw, weight_raw), metric, log

    items = list(enumerate(images, 1))
    workers = max(1, min(int(preprocess_workers), len(items))) if items else 1
    if workers == 1:
        results = [prepare_one(it) for it in items]
    else:
        with ThreadPoolExecutor(max_workers=workers) as pool:
            results = list(pool.map(prepare_one, items))
    prepared, metrics = [], []
    for pair, metric, log in results:
        prepared.append(pair)
        metrics.append(metric)
        print(log, flush=True)
    return prepared, metrics
