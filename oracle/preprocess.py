"""TEST INFRASTRUCTURE ONLY — CPU restatement of the reference's per-exposure
weight preprocessing (updc/_engine.py:287-408 of the reference).

Only ``tests/`` and bench.py's CPU-baseline leg may import this module; the
product path (``updc_b200.preprocess``) runs on the GPU and never calls it.

What is restated, step by step, in the reference's numeric types (NumPy 2
semantics: a Python float compared with a float32 array is rounded to
float32 first; a float32 median of an even count is the float32 mean of the
two middle order statistics):

* ``robust_background_mask`` (_engine.py:287-310): asymmetric sigma clipping
  of SCI over the base-valid pixels, at most 6 passes, window
  (med - 4.5 sig, med + 2.5 sig) with sig = 1.4826 MAD, falling back to the
  float32 standard deviation when the MAD is zero, stopping when the mask
  repeats; then the final median and 1.4826 MAD (a float32 product there).
* ``build_weight`` (_engine.py:313-333): sky VAR_POISSON median and the three
  weight modes in float64.
* the numeric part of ``prepare_weighted_inputs.prepare_one``
  (_engine.py:349-397): base-valid mask, usable mask, automatic and
  requested pedestals, the positivity check, the float32 WHT plane and the
  metrics record.

The float32 standard deviation follows NumPy's own reduction order (pairwise
summation: blocks of at most 128 values summed with eight interleaved
accumulators, halves split at multiples of eight; the mean and variance
divisions done in float64 and rounded to float32), so the fallback threshold
is reproduced exactly; ``std_f32`` is checked against ``numpy.std``.

Pinned: ``tests/golden/preprocess/`` holds outputs of the reference's own
functions (generated by ``tests/golden/make_preprocess_golden.py``), and the
tests compare this restatement with them.
"""
from __future__ import annotations

import numpy as np

MAX_ITER = 6
CLIP_LOW, CLIP_HIGH = 4.5, 2.5
MAD_TO_SIGMA = 1.4826
WEIGHT_MODES = ("mask", "rnoise-sky", "totalvar")


class PreprocessError(ValueError):
    """The reference raises ValueError with these messages."""


# ----------------------------------------------------------------------------- order statistics
def median(vals: np.ndarray):
    """numpy.median of a 1-D array in its own dtype (nan when empty)."""
    t = vals.dtype.type
    m = vals.size
    if m == 0:
        return t(np.nan)
    hi = m // 2
    if m % 2:
        return np.partition(vals, hi)[hi]
    part = np.partition(vals, [hi - 1, hi])
    return t(t(part[hi - 1] + part[hi]) / t(2))


# ----------------------------------------------------------------------------- NumPy's float32 sum order
PAIRWISE_BLOCK = 128


def _block_sum(a: np.ndarray) -> np.float32:
    f = np.float32
    n = a.size
    if n < 8:
        s = f(-0.0)
        for v in a:
            s = f(s + v)
        return s
    acc = a[:8].copy()
    tail = n - n % 8
    for i in range(8, tail, 8):
        acc = acc + a[i:i + 8]
    s = f(f(f(acc[0] + acc[1]) + f(acc[2] + acc[3])) + f(f(acc[4] + acc[5]) + f(acc[6] + acc[7])))
    for v in a[tail:]:
        s = f(s + v)
    return s


def pairwise_sum_f32(a: np.ndarray) -> np.float32:
    """Sum of a float32 vector in NumPy's pairwise order."""
    a = np.ascontiguousarray(a, dtype=np.float32)

    def rec(lo: int, n: int) -> np.float32:
        if n <= PAIRWISE_BLOCK:
            return _block_sum(a[lo:lo + n])
        half = n // 2
        half -= half % 8
        return np.float32(rec(lo, half) + rec(lo + half, n - half))

    return np.float32(np.float32(-0.0) + rec(0, a.size))


def std_f32(vals: np.ndarray) -> np.float32:
    """numpy.std of a float32 vector (ddof 0), restated."""
    n = vals.size
    mean = np.float32(np.float64(pairwise_sum_f32(vals)) / np.float64(n))
    dev = vals - mean
    dev = dev * dev
    var = np.float32(np.float64(pairwise_sum_f32(dev)) / np.float64(n))
    return np.sqrt(var)


# ----------------------------------------------------------------------------- _engine.py:287-310
def clip_window(science: np.ndarray, base_valid: np.ndarray, med: float, sig: float) -> np.ndarray:
    lo = np.float32(med - CLIP_LOW * sig)
    hi = np.float32(med + CLIP_HIGH * sig)
    return base_valid & (science > lo) & (science < hi)


def robust_background(science: np.ndarray, base_valid: np.ndarray, max_iter: int = MAX_ITER):
    """Returns (mask, background, sigma, passes, std_fallbacks)."""
    need = max(32, min(1000, base_valid.size // 100))
    mask = base_valid.copy()
    passes = fallbacks = 0
    for _ in range(max_iter):
        vals = science[mask]
        if vals.size < need:
            raise PreprocessError("Too few valid pixels for robust background estimation")
        med = float(median(vals))
        sig = MAD_TO_SIGMA * float(median(np.abs(vals - np.float32(med))))
        if not (np.isfinite(sig) and sig > 0):
            fallbacks += 1
            sig = float(std_f32(vals))
        if not (np.isfinite(sig) and sig > 0):
            raise PreprocessError("Cannot estimate a positive background RMS")
        passes += 1
        new = clip_window(science, base_valid, med, sig)
        same = np.array_equal(new, mask)
        mask = new
        if same:
            break
    vals = science[mask]
    med = float(median(vals))
    # here the MAD stays a float32 scalar, so the scale factor is rounded to
    # float32 and the product is a float32 product (inside the loop the MAD
    # is a Python float and the product is float64)
    sig = float(np.float32(MAD_TO_SIGMA) * median(np.abs(vals - np.float32(med))))
    return mask, med, sig, passes, fallbacks


# ----------------------------------------------------------------------------- _engine.py:313-333
def sky_var_poisson(var_p: np.ndarray, sky_mask: np.ndarray) -> float:
    sel = sky_mask & np.isfinite(var_p) & (var_p >= 0)
    v = float(median(var_p[sel]))
    if not np.isfinite(v) or v < 0:
        raise PreprocessError("Cannot estimate sky VAR_POISSON")
    return v


def raw_weight(mode: str, var_p, var_r, var_f, sky_var_p: float) -> np.ndarray:
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        if mode == "mask":
            return np.ones_like(var_r, dtype=np.float64)
        if mode == "rnoise-sky":
            return 1.0 / (var_r + sky_var_p)
        if mode == "totalvar":
            return 1.0 / ((var_p + var_r) + var_f)
    raise PreprocessError(mode)


# ----------------------------------------------------------------------------- _engine.py:349-397
def prepare_exposure(science, dq, var_p, var_r, var_f, weight_mode: str, bad_dq_mask: int,
                     pedestal_sigma: float, source: str = ""):
    """Returns (wht float32, metrics dict, passes, std_fallbacks)."""
    science = np.asarray(science, dtype=np.float32)
    dq = np.asarray(dq, dtype=np.uint32)
    var_p, var_r, var_f = (np.asarray(v, dtype=np.float64) for v in (var_p, var_r, var_f))
    base_valid = np.isfinite(science) & ((dq & np.uint32(bad_dq_mask)) == 0)
    base_valid &= np.isfinite(var_p) & np.isfinite(var_r)
    if weight_mode == "totalvar":
        base_valid &= np.isfinite(var_f)
    sky_mask, background, sky_sigma, passes, fallbacks = robust_background(science, base_valid)
    svp = sky_var_poisson(var_p, sky_mask)
    w = raw_weight(weight_mode, var_p, var_r, var_f, svp)
    usable = base_valid & np.isfinite(w) & (w > 0)
    if not usable.any():
        raise PreprocessError(f"No usable pixels remain in {source}")
    min_valid = float(np.min(science[usable]))
    floor = max(1.0e-12, 1.0e-6 * sky_sigma)
    auto = max(0.0, floor - min_valid)
    requested = max(0.0, pedestal_sigma * sky_sigma - background)
    pedestal = max(auto, requested)
    before = int((usable & (science <= 0)).sum())
    after = int((usable & (science.astype(np.float64) + pedestal <= 0)).sum())
    if after:
        raise PreprocessError(f"Automatic pedestal failed to make y_eff positive in {source}")
    wht = np.where(usable, w, 0.0).astype(np.float32)
    if not (wht > 0).any():
        raise PreprocessError(f"No usable pixels remain in {source}")
    metrics = {
        "background": background, "background_sigma": sky_sigma, "poisson_pedestal": pedestal,
        "auto_positivity_pedestal": auto, "requested_pedestal": requested, "min_valid_science": min_valid,
        "sky_var_poisson": svp, "weight_mode": weight_mode, "base_invalid": int((~base_valid).sum()),
        "nonpositive_valid_before_pedestal": before, "nonpositive_after_pedestal": after,
        "wht_zero": int((wht == 0).sum()), "wht_valid_median": float(median(wht[wht > 0])),
    }
    return wht, metrics, passes, fallbacks
