"""Seeded synthetic inputs in the reference engine-handoff format.

The reference measures on JWST data that is not distributed with it, so every
workload here is synthetic.  ``generate`` writes exactly the file set that
updc/_engine.py hands the frozen core (manifest TSV, raw float32 SCI/WHT/PSF,
float64 vertex maps; see ``updc_b200.handoff``) for a named workload:

* ``c0``    256^2 target, 4 x 128^2 detectors, 33^2 Gaussian+Moffat PSF
            (the reference's CPU-runnable case);
* ``c1``    4096^2 target, 8 x 2048^2 detectors with affine + cubic
            distortion, 1431^2 hexagonal-pupil PSF per exposure (the headline);
* ``c3``    2048^2 target, 4 x 1024^2 detectors, 1431^2 Gaussian+Moffat PSF;
* ``c4``    8192^2 target, 16 x 4096^2 detectors, 1431^2 hexagonal PSF;
* ``small`` / ``medium`` / ``abs32`` reduced cases used by the parity tests
            (``abs32`` is 66000 target pixels wide, so detector stencils span
            more than 65535 indices and force the ABS32 LinkMap encoding).

Detector data are Poisson(H x + background) + N(0, 5^2) with W = 1/variance.
H x is approximated here by PSF convolution followed by a 4-point quadrature of
each mapped detector pixel; data only need to be realistic, not exact, because
every solver (reference, oracle, GPU) consumes the same files.  The pedestal is
``max(10, 1e-6 * sigma_read - min(SCI))`` per exposure, the reference's
automatic-pedestal rule (updc/_engine.py:364-369), so that y_eff = SCI +
pedestal is positive as the core requires (updc_core.c:370-371).  A small
fraction of SCI pixels is set to NaN to exercise the invalid-pixel mask
(updc_core.c:365-367).
"""
from __future__ import annotations

import dataclasses
import math
import os
from pathlib import Path
from typing import Dict, List, Optional

import numpy as np

from .handoff import EngineArgs, ExposureRow, write_manifest


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    W: int
    H: int
    iw: int
    ih: int
    nexp: int
    psf_size: int
    psf_kind: str            # "gauss_moffat" or "hex"
    n_points: int
    n_galaxies: int
    iterations: int
    scale: float = 2.0       # target pixels per detector pixel
    dither_max: float = 2.0
    distortion: bool = False
    point_flux_max: float = 1.0e4
    sky: float = 0.3
    background: float = 0.3
    read_noise: float = 5.0
    bad_fraction: float = 1.0e-3
    psf_sigma: float = 1.2
    seed: int = 0


WORKLOADS: Dict[str, Workload] = {
    "c0": Workload("c0", 256, 256, 128, 128, 4, 33, "gauss_moffat", 40, 10, 20),
    "c1": Workload("c1", 4096, 4096, 2048, 2048, 8, 1431, "hex", 20000, 2000, 39,
                   dither_max=10.0, distortion=True, bad_fraction=1.0e-4),
    "c3": Workload("c3", 2048, 2048, 1024, 1024, 4, 1431, "gauss_moffat", 5000, 500, 10,
                   dither_max=10.0, distortion=True, bad_fraction=1.0e-4),
    "c4": Workload("c4", 8192, 8192, 4096, 4096, 16, 1431, "hex", 80000, 8000, 39,
                   dither_max=10.0, distortion=True, point_flux_max=1.0e6, bad_fraction=1.0e-4),
    "small": Workload("small", 96, 80, 44, 36, 3, 15, "gauss_moffat", 12, 3, 4, seed=3),
    "medium": Workload("medium", 512, 512, 256, 256, 4, 65, "gauss_moffat", 200, 40, 6,
                       dither_max=4.0, distortion=True, seed=1),
    # detector pixels 20 target pixels tall: a stencil spans ~20 rows of a
    # 3400-wide grid (> 65535 indices), forcing ABS32 on a grid the engine's
    # single-block row transform holds
    "abs32": Workload("abs32", 3400, 48, 6, 2, 2, 3, "gauss_moffat", 3, 0, 2,
                      scale=20.0, dither_max=0.5, seed=5),
    # the reference's own ABS32 validation geometry (target width 70000 class);
    # (rows of 33075 complex points: the GPU engine's four-step long-row path)
    "abs32_wide": Workload("abs32_wide", 66000, 6, 6, 2, 2, 3, "gauss_moffat", 3, 0, 2,
                           scale=2.0, dither_max=0.5, seed=5),
}


@dataclasses.dataclass
class Dataset:
    workload: Workload
    directory: Path
    manifest: Path
    rows: List[ExposureRow]

    def engine_args(self, iterations: Optional[int] = None, prefix: str = "iter",
                    save_every: int = 0, **kw) -> EngineArgs:
        w = self.workload
        return EngineArgs(str(self.manifest), w.W, w.H, w.iw, w.ih, w.nexp, 0,
                          iterations if iterations is not None else w.iterations,
                          str(self.directory / prefix), str(self.directory / f"{prefix}_wht.bin"),
                          save_every=save_every, **kw)


# ----------------------------------------------------------------------------- PSFs

def gauss_moffat_psf(size: int, sigma: float = 1.2, beta: float = 2.5, alpha: float = 3.0,
                     wing: float = 0.05) -> np.ndarray:
    c = (size - 1) / 2.0
    yy, xx = np.indices((size, size), dtype=np.float64)
    r2 = (xx - c) ** 2 + (yy - c) ** 2
    g = np.exp(-r2 / (2.0 * sigma * sigma))
    m = (1.0 + r2 / (alpha * alpha)) ** (-beta)
    psf = (1.0 - wing) * g / g.sum() + wing * m / m.sum()
    return (psf / psf.sum()).astype(np.float32)


def hex_pupil_psf(size: int, rng: np.random.Generator, grid: int = 2048,
                  oversample: float = 4.0, rms_nm: float = 20.0, wavelength_nm: float = 2000.0,
                  use_torch: bool = False) -> np.ndarray:
    """|FFT|^2 of an 18-segment hexagonal pupil with random segment phases.

    Segments are flat-topped hexagons on the two rings around a missing centre
    (axial coordinates |q|,|r|,|q+r| <= 2 without (0,0)).  Each segment gets a
    random piston, tip and tilt with ``rms_nm`` rms wavefront at
    ``wavelength_nm``.  The PSF is sampled at 1/oversample of lambda/D.
    """
    aperture = grid / oversample                     # pupil diameter in grid pixels
    rs = aperture / (5.0 * math.sqrt(3.0))           # segment circumradius
    yy, xx = np.indices((grid, grid), dtype=np.float64)
    u0 = xx - grid / 2.0
    v0 = yy - grid / 2.0
    phase = np.zeros((grid, grid))
    pupil = np.zeros((grid, grid))
    rad = 2.0 * math.pi * rms_nm / wavelength_nm
    for q in range(-2, 3):
        for r in range(-2, 3):
            if abs(q + r) > 2 or (q == 0 and r == 0):
                continue
            cx = rs * 1.5 * q
            cy = rs * math.sqrt(3.0) * (r + q / 2.0)
            u = u0 - cx
            v = v0 - cy
            shrink = 0.97 * rs
            inside = (np.abs(v) <= math.sqrt(3.0) / 2.0 * shrink) & \
                     (math.sqrt(3.0) * np.abs(u) + np.abs(v) <= math.sqrt(3.0) * shrink)
            piston, tip, tilt = rng.normal(0.0, rad, 3)
            pupil[inside] = 1.0
            phase[inside] = piston + tip * u[inside] / rs + tilt * v[inside] / rs
    field = pupil * np.exp(1j * phase)
    if use_torch:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        f = torch.fft.fftshift(torch.fft.fft2(torch.from_numpy(field).to(dev)))
        img = (f.real ** 2 + f.imag ** 2).cpu().numpy()
    else:
        f = np.fft.fftshift(np.fft.fft2(field))
        img = f.real ** 2 + f.imag ** 2
    c = grid // 2
    h = size // 2
    crop = img[c - h:c - h + size, c - h:c - h + size]
    return (crop / crop.sum()).astype(np.float32)


# ----------------------------------------------------------------------------- scene

def sersic_b(n: float) -> float:
    return 2.0 * n - 1.0 / 3.0 + 4.0 / (405.0 * n) + 46.0 / (25515.0 * n * n)


def render_scene(w: Workload, rng: np.random.Generator) -> np.ndarray:
    img = np.full((w.H, w.W), w.sky, dtype=np.float64)
    # point sources: log-uniform flux, bilinear splat at sub-pixel positions
    n = w.n_points
    if n:
        px = rng.uniform(0, w.W - 1, n)
        py = rng.uniform(0, w.H - 1, n)
        flux = np.exp(rng.uniform(math.log(10.0), math.log(w.point_flux_max), n))
        x0 = np.floor(px).astype(np.int64)
        y0 = np.floor(py).astype(np.int64)
        fx = px - x0
        fy = py - y0
        for dy, dx, wgt in ((0, 0, (1 - fx) * (1 - fy)), (0, 1, fx * (1 - fy)),
                            (1, 0, (1 - fx) * fy), (1, 1, fx * fy)):
            xi = np.minimum(x0 + dx, w.W - 1)
            yi = np.minimum(y0 + dy, w.H - 1)
            np.add.at(img, (yi, xi), flux * wgt)
    # Sersic galaxies
    for _ in range(w.n_galaxies):
        cx = rng.uniform(0, w.W - 1)
        cy = rng.uniform(0, w.H - 1)
        nser = rng.uniform(0.5, 4.0)
        re = rng.uniform(2.0, 12.0)
        q = rng.uniform(0.4, 1.0)
        pa = rng.uniform(0.0, math.pi)
        flux = math.exp(rng.uniform(math.log(100.0), math.log(1.0e4)))
        half = int(min(6.0 * re + 3.0, 96.0))
        xa, xb = max(0, int(cx) - half), min(w.W, int(cx) + half + 1)
        ya, yb = max(0, int(cy) - half), min(w.H, int(cy) + half + 1)
        if xa >= xb or ya >= yb:
            continue
        yy, xx = np.mgrid[ya:yb, xa:xb].astype(np.float64)
        dx = xx - cx
        dy = yy - cy
        c, s = math.cos(pa), math.sin(pa)
        u = dx * c + dy * s
        v = -dx * s + dy * c
        r = np.sqrt(u * u + (v / q) ** 2)
        prof = np.exp(-sersic_b(nser) * ((r / re) ** (1.0 / nser) - 1.0))
        tot = prof.sum()
        if tot > 0:
            img[ya:yb, xa:xb] += flux * prof / tot
    return img


# ----------------------------------------------------------------------------- geometry

def detector_vertices(w: Workload, rng: np.random.Generator) -> np.ndarray:
    """(ih+1, iw+1, 2) float64 target coordinates of detector pixel corners."""
    theta = math.radians(rng.uniform(-3.0, 3.0))
    s = rng.uniform(0.99, 1.01)
    shear = rng.uniform(-0.005, 0.005)
    dither = rng.uniform(0.0, w.dither_max, 2)
    rot = np.array([[math.cos(theta), -math.sin(theta)], [math.sin(theta), math.cos(theta)]])
    a = w.scale * s * rot @ np.array([[1.0, shear], [0.0, 1.0]])
    yy, xx = np.indices((w.ih + 1, w.iw + 1), dtype=np.float64)
    dx = (xx - 0.5) - (w.iw - 1) / 2.0
    dy = (yy - 0.5) - (w.ih - 1) / 2.0
    if w.distortion:
        # quadratic (~1e-6 px^-1) plus cubic (~1e-10 px^-2) polynomial terms, a
        # displacement of at most a couple of detector pixels at the corners
        c2 = rng.normal(0.0, 1.0e-6, 6)
        c3 = rng.normal(0.0, 1.0e-10, 4)
        ddx = c2[0] * dx * dx + c2[1] * dx * dy + c2[2] * dy * dy + c3[0] * dx ** 3 + c3[1] * dx * dy * dy
        ddy = c2[3] * dx * dx + c2[4] * dx * dy + c2[5] * dy * dy + c3[2] * dy ** 3 + c3[3] * dx * dx * dy
        dx = dx + ddx
        dy = dy + ddy
    ctx = (w.W - 1) / 2.0 + dither[0] - w.dither_max / 2.0
    cty = (w.H - 1) / 2.0 + dither[1] - w.dither_max / 2.0
    tx = ctx + a[0, 0] * dx + a[0, 1] * dy
    ty = cty + a[1, 0] * dx + a[1, 1] * dy
    return np.stack((tx, ty), axis=-1)


def _blur(scene: np.ndarray, psf: np.ndarray, use_torch: bool) -> np.ndarray:
    """Linear convolution with the PSF centre at (ph//2, pw//2), cropped to the
    scene (the convention of updc_core.c:816-821)."""
    H, W = scene.shape
    ph, pw = psf.shape
    fh, fw = H + ph - 1, W + pw - 1
    kern = np.zeros((fh, fw))
    ys = (np.arange(ph) - ph // 2) % fh
    xs = (np.arange(pw) - pw // 2) % fw
    kern[np.ix_(ys, xs)] = psf
    if use_torch:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        a = torch.zeros((fh, fw), dtype=torch.float64, device=dev)
        a[:H, :W] = torch.from_numpy(scene).to(dev)
        k = torch.from_numpy(kern).to(dev)
        out = torch.fft.irfft2(torch.fft.rfft2(a) * torch.fft.rfft2(k), s=(fh, fw))
        return out[:H, :W].cpu().numpy()
    a = np.zeros((fh, fw))
    a[:H, :W] = scene
    out = np.fft.irfft2(np.fft.rfft2(a) * np.fft.rfft2(kern), s=(fh, fw))
    return out[:H, :W]


def _sample(img: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Bilinear sample with zero outside the grid."""
    H, W = img.shape
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    fx = x - x0
    fy = y - y0
    out = np.zeros(x.shape)
    for dy, dx, wgt in ((0, 0, (1 - fx) * (1 - fy)), (0, 1, fx * (1 - fy)),
                        (1, 0, (1 - fx) * fy), (1, 1, fx * fy)):
        xi = x0 + dx
        yi = y0 + dy
        ok = (xi >= 0) & (xi < W) & (yi >= 0) & (yi < H)
        out[ok] += wgt[ok] * img[yi[ok], xi[ok]]
    return out


def generate(name_or_workload, directory: os.PathLike, use_torch: Optional[bool] = None) -> Dataset:
    """Write the handoff file set for a workload into ``directory``."""
    w = WORKLOADS[name_or_workload] if isinstance(name_or_workload, str) else name_or_workload
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    if use_torch is None:
        use_torch = w.W * w.H > 1024 * 1024
    rng = np.random.default_rng(w.seed)
    scene = render_scene(w, rng)
    rows: List[ExposureRow] = []
    shared_psf = None
    for k in range(1, w.nexp + 1):
        if w.psf_kind == "hex":
            psf = hex_pupil_psf(w.psf_size, rng, use_torch=use_torch)
        else:
            if shared_psf is None:
                shared_psf = gauss_moffat_psf(w.psf_size, sigma=w.psf_sigma)
            psf = shared_psf
        verts = detector_vertices(w, rng)
        blurred = _blur(scene, psf.astype(np.float64), use_torch)
        # 4-point quadrature of the mapped pixel (midpoints of its quadrants)
        c00, c01 = verts[:-1, :-1], verts[:-1, 1:]
        c10, c11 = verts[1:, :-1], verts[1:, 1:]
        model = np.zeros((w.ih, w.iw))
        for a, b in ((0.25, 0.25), (0.75, 0.25), (0.25, 0.75), (0.75, 0.75)):
            p = ((1 - a) * (1 - b)) * c00 + (a * (1 - b)) * c01 + ((1 - a) * b) * c10 + (a * b) * c11
            model += 0.25 * _sample(blurred, p[..., 0], p[..., 1])
        mean = model + w.background
        counts = rng.poisson(np.maximum(mean, 0.0)).astype(np.float64)
        sci = counts + rng.normal(0.0, w.read_noise, mean.shape)
        wht = 1.0 / (np.maximum(mean, 0.0) + w.read_noise ** 2)
        sci = sci.astype(np.float32)
        wht = wht.astype(np.float32)
        if w.bad_fraction > 0:
            nbad = max(1, int(w.bad_fraction * sci.size))
            bad = rng.choice(sci.size, nbad, replace=False)
            sci.reshape(-1)[bad] = np.nan
        valid = np.isfinite(sci) & (wht > 0)
        floor = max(1.0e-12, 1.0e-6 * w.read_noise)
        pedestal = max(10.0, floor - float(np.min(sci[valid].astype(np.float64))))
        files = {n: d / f"{n}_{k}.{ext}" for n, ext in
                 (("science", "f32"), ("weight", "f32"), ("psf", "f32"), ("vertices", "bin"))}
        sci.astype("<f4").tofile(files["science"])
        wht.astype("<f4").tofile(files["weight"])
        psf.astype("<f4").tofile(files["psf"])
        verts.astype("<f8").tofile(files["vertices"])
        rows.append(ExposureRow(str(files["science"]), str(files["weight"]), str(files["psf"]),
                                psf.shape[1], psf.shape[0], str(files["vertices"]),
                                w.background, pedestal))
    manifest = d / "manifest.txt"
    write_manifest(manifest, rows)
    return Dataset(w, d, manifest, rows)


# ----------------------------------------------------------------------------- batched cutouts
BATCH_GRIDS = (128, 192, 256, 384, 512, 768)


def batch_workloads(n_fields: int = 64, seed: int = 2, iterations: int = 30) -> List[Workload]:
    """Independent cutout fields: target grid uniform over BATCH_GRIDS (square),
    3-12 exposures of target/2 +- 16 detector pixels at scale 2 with random
    affine maps and dithers as in c0, Gaussian+Moffat PSFs of 33-129 px with a
    core width of 1.0-1.6 px; scene density as c0 per unit area."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_fields):
        t = int(rng.choice(BATCH_GRIDS))
        nexp = int(rng.integers(3, 13))
        det = t // 2 + int(rng.integers(-16, 17))
        psf = 2 * int(rng.integers(16, 65)) + 1
        area = (t / 256.0) ** 2
        out.append(Workload(f"field{i:02d}", t, t, det, det, nexp, psf, "gauss_moffat",
                            max(4, int(40 * area)), max(1, int(10 * area)), iterations,
                            psf_sigma=float(rng.uniform(1.0, 1.6)), seed=1000 + i))
    return out


def generate_batch(directory: os.PathLike, n_fields: int = 64, seed: int = 2,
                   iterations: int = 30) -> List[Dataset]:
    """Write one handoff file set per field under ``directory/<field name>``."""
    d = Path(directory)
    return [generate(w, d / w.name, use_torch=False) for w in batch_workloads(n_fields, seed, iterations)]


# ----------------------------------------------------------------------------- PSF projection cases
def psf_projection_case(directory: os.PathLike, name: str, size: int, oversample: int, seed: int,
                        distortion: float = 1.0e-4):
    """An oversampled Gaussian+Moffat PSF (size x size, odd) and the target
    offsets of its pixel corners: a detector-pixel offset (i - size/2) /
    oversample mapped by 2 x rotation x scale x shear plus a quadratic
    distortion, centred on the PSF centre (the layout of _engine.py:470-521's
    vertex files).  Writes <name>.f32 and <name>.vertices.bin; returns their
    paths."""
    rng = np.random.default_rng(seed)
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    psf = gauss_moffat_psf(size, sigma=float(rng.uniform(1.0, 2.5)))
    g = (np.arange(size + 1, dtype=np.float64) - size / 2.0) / float(oversample)
    xx, yy = np.meshgrid(g, g)
    th = np.deg2rad(rng.uniform(-30.0, 30.0))
    s = 2.0 * rng.uniform(0.98, 1.02)
    sh = rng.uniform(-0.01, 0.01)
    A = s * np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]]) @ np.array([[1.0, sh], [0.0, 1.0]])
    px = A[0, 0] * xx + A[0, 1] * yy + distortion * (xx * xx - yy * yy)
    py = A[1, 0] * xx + A[1, 1] * yy + distortion * 2.0 * xx * yy
    f_psf = d / f"{name}.f32"
    f_vert = d / f"{name}.vertices.bin"
    psf.astype("<f4").tofile(f_psf)
    np.stack((px, py), axis=-1).astype("<f8").tofile(f_vert)
    return f_psf, f_vert



# ----------------------------------------------------------------------------- Level-2 exposures (weights)
# Each case: (shape, weight_mode, bad_dq_mask, pedestal_sigma, pattern).  The
# patterns exercise the branches of the per-exposure preprocessing: sources
# above a noisy sky with bad DQ bits and non-finite pixels, each weight mode,
# a requested pedestal, ties and an even number of clipped pixels, a MAD of
# zero (standard-deviation fallback), and every failure the reference raises.
PREPROCESS_CASES = {
    "sky_sources": ((32, 40), "rnoise-sky", 1, 0.0, "sources"),
    "totalvar_requested": ((48, 36), "totalvar", 5, 3.0, "sources"),
    "mask_negative_sky": ((40, 40), "mask", 1, 0.0, "negative"),
    "integer_ties": ((30, 44), "rnoise-sky", 1, 0.0, "ties"),
    "mad_zero": ((36, 36), "rnoise-sky", 1, 0.0, "mad_zero"),
    "too_few_valid": ((32, 32), "rnoise-sky", 1, 0.0, "too_few"),
    "no_background_rms": ((32, 32), "rnoise-sky", 1, 0.0, "constant"),
    "no_sky_var": ((32, 32), "rnoise-sky", 1, 0.0, "negative_var_p"),
    "no_usable": ((32, 32), "rnoise-sky", 1, 0.0, "negative_var_r"),
    "weight_underflow": ((32, 32), "rnoise-sky", 1, 0.0, "huge_var_r"),
    "pedestal_fails": ((32, 32), "mask", 1, 0.0, "huge_negative"),
    "unknown_mode": ((32, 32), "inverse-variance", 1, 0.0, "sources"),
}


def level2_exposure(shape, pattern: str, seed: int) -> dict:
    """Synthetic Level-2 planes: SCI (f32), DQ (u32), VAR_POISSON, VAR_RNOISE,
    VAR_FLAT (f32 as stored in the files; the preprocessing reads them as f64)."""
    rng = np.random.default_rng(seed)
    h, w = shape
    n = h * w
    sky = float(rng.uniform(0.2, 2.0))
    rms = float(rng.uniform(0.5, 5.0))
    sci = sky + rms * rng.standard_normal(n)
    nsrc = max(1, n // 80)
    idx = rng.choice(n, nsrc, replace=False)
    sci[idx] += 10.0 ** rng.uniform(1.0, 4.0, nsrc)
    dq = np.zeros(n, np.uint32)
    dq[rng.choice(n, n // 50, replace=False)] = rng.choice([1, 2, 4, 1024], n // 50).astype(np.uint32)
    var_p = np.abs(sci) * 1e-3 + 1e-4
    var_r = np.full(n, rms * rms) * rng.uniform(0.9, 1.1, n)
    var_f = np.full(n, 1e-4) * rng.uniform(0.5, 1.5, n)
    if pattern == "negative":
        sci -= 3.0 * sky + 4.0 * rms
    elif pattern == "ties":
        sci = np.round(sci)
    elif pattern == "mad_zero":
        sci[rng.random(n) < 0.6] = 2.0
    elif pattern == "too_few":
        dq[:] = 1
        dq[rng.choice(n, 20, replace=False)] = 0
    elif pattern == "constant":
        sci[:] = 1.5
    elif pattern == "negative_var_p":
        var_p[:] = -1.0
    elif pattern == "negative_var_r":
        var_r[:] = -1.0e9
    elif pattern == "huge_var_r":
        var_r[:] = 1.0e300
    elif pattern == "huge_negative":
        sci[rng.integers(n)] = -1.0e20
    sci = sci.astype(np.float32)
    nonfinite = rng.choice(n, max(1, n // 200), replace=False)
    if pattern not in ("constant", "too_few"):
        sci[nonfinite[: len(nonfinite) // 2 + 1]] = np.nan
        var_f[nonfinite[len(nonfinite) // 2:]] = np.inf
    planes = {"SCI": sci, "DQ": dq, "VAR_POISSON": var_p.astype(np.float32), "VAR_RNOISE": var_r.astype(np.float64),
              "VAR_FLAT": var_f.astype(np.float32)}
    return {k: v.reshape(h, w) for k, v in planes.items()}


def preprocess_case(name: str, index: int = 1) -> dict:
    shape, _mode, _dqmask, _ped, pattern = PREPROCESS_CASES[name]
    seed = 1000 + 17 * sorted(PREPROCESS_CASES).index(name) + index
    return level2_exposure(shape, pattern, seed)
