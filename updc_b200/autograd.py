"""Differentiable UPDC forward model: sum_k H_k and the weighted Poisson NLL
as a ``torch.autograd.Function``.

The reference's multiplicative update (updc/c_core/updc_core.c:1437-1456)
is the fixed-point step of the weighted Poisson likelihood of its forward
model (core:1140-1183).  This module exposes that likelihood to autograd:

    mu_k = S_k P_k x + background_k + pedestal_k        (raw_mu, core:1152-1160)
    y_k  = SCI_k + pedestal_k                           (y_eff, core:1161)
    L    = sum_k sum_p W_kp (mu_kp - y_kp log mu_kp)    (W > 0, mu > 0)

with hand-written CUDA for both directions (``updc_nll`` and
``updc_nll_adjoint`` of the C ABI): the backward of x is
sum_k P_k^T S_k^T r_k with r = W (1 - y/mu), i.e. the engine's transposed
gather and conj-OTF adjoint run on r instead of W * ratio.  Gradients also
flow to the per-exposure background and pedestal (reductions of r and
W log mu) and to the PSFs (the cross-correlation of S_k^T r_k with x on the
PSF window), so a parametric PSF such as ``gauss_moffat_psf`` with a
Gaussian width sigma gets d L / d sigma through torch.  The backward
recomputes the forward planes from the saved inputs; nothing but the inputs
is kept between forward and backward.

PyTorch tensors appear only here, at the autograd boundary: x goes to the
engine by a device-to-device copy, everything else through the C ABI.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .engine import Engine


def gauss_moffat_psf(size: int, sigma, beta: float = 2.5, alpha: float = 3.0, wing: float = 0.05,
                     dtype=torch.float64) -> torch.Tensor:
    """Gaussian core of width ``sigma`` plus a Moffat wing, normalised to sum 1
    (the same model as ``synth.gauss_moffat_psf``), differentiable in sigma."""
    sigma = torch.as_tensor(sigma, dtype=dtype)
    c = (size - 1) / 2.0
    yy, xx = torch.meshgrid(torch.arange(size, dtype=dtype), torch.arange(size, dtype=dtype), indexing="ij")
    r2 = (xx - c) ** 2 + (yy - c) ** 2
    g = torch.exp(-r2 / (2.0 * sigma * sigma))
    m = (1.0 + r2 / (alpha * alpha)) ** (-beta)
    psf = (1.0 - wing) * g / g.sum() + wing * m / m.sum()
    return psf / psf.sum()


class PoissonModel:
    """An engine set up on one field (manifest + geometry) whose estimate,
    per-exposure background/pedestal and PSFs are inputs of the likelihood."""

    def __init__(self, manifest: str, width: int, height: int, input_width: int, input_height: int,
                 exposures: int, form: str = "fp32", device: int = 0, **engine_kw):
        self.engine = Engine(form=form, device=device, use_graph=False, **engine_kw)
        self.engine.load(manifest, width, height, input_width, input_height, exposures).setup()
        self.form = form
        self.nexp = exposures
        self.shape = (height, width)
        self.dtype = torch.float64 if form == "fp64" else torch.float32
        self.device = torch.device("cuda", device)

    def close(self) -> None:
        self.engine.close()

    def _load(self, x: torch.Tensor, background: torch.Tensor, pedestal: torch.Tensor,
              psf: Optional[torch.Tensor]) -> Optional[np.ndarray]:
        """Inputs -> engine state; returns the PSFs as FP64 host arrays (or None)."""
        if tuple(x.shape) != self.shape or not x.is_cuda:
            raise ValueError(f"x must be a CUDA tensor of shape {self.shape}")
        xc = x.detach().contiguous()
        if xc.dtype not in (torch.float32, torch.float64):
            xc = xc.to(self.dtype)
        self.engine.copy_plane_device("estimate", xc.data_ptr(), to_engine=True, as_double=xc.dtype == torch.float64,
                                      stream=torch.cuda.current_stream(x.device).cuda_stream)
        b = background.detach().double().cpu().numpy()
        p = pedestal.detach().double().cpu().numpy()
        for k in range(self.nexp):
            self.engine.set_exposure_offsets(k, float(b[k]), float(p[k]))
        if psf is None:
            return None
        ps = psf.detach().double().cpu().numpy()
        for k in range(self.nexp):
            self.engine.set_psf(k, ps[k])
        return ps

    def loss(self, x, background, pedestal, psf=None) -> torch.Tensor:
        return PoissonNLL.apply(x, background, pedestal, psf, self)

    def terms(self) -> np.ndarray:
        """Per-exposure [L_k, sum r, sum W log mu, pixels left out] of the current inputs."""
        return self.engine.nll()


class PoissonNLL(torch.autograd.Function):
    """L(x, background, pedestal, psf) of a ``PoissonModel``; ``psf`` may be
    None (the manifest PSFs, no PSF gradient) or an (N, ph, pw) tensor of raw
    PSFs, which the engine normalises by their sums."""

    @staticmethod
    def forward(ctx, x, background, pedestal, psf, model: PoissonModel):
        model._load(x, background, pedestal, psf)
        terms = model.engine.nll()
        ctx.model = model
        ctx.has_psf = psf is not None
        ctx.save_for_backward(x, background, pedestal, psf if psf is not None else torch.empty(0))
        return torch.tensor(float(terms[:, 0].sum()), dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, grad):
        model: PoissonModel = ctx.model
        x, background, pedestal, psf = ctx.saved_tensors
        ps = model._load(x, background, pedestal, psf if ctx.has_psf else None)
        terms = model.engine.nll()          # recompute the forward planes and r
        model.engine.nll_adjoint()           # CORRECTION <- sum_k H_k^T r_k
        g = float(grad)
        gx = torch.empty(x.shape, dtype=x.dtype if x.dtype in (torch.float32, torch.float64) else model.dtype,
                         device=x.device)
        model.engine.copy_plane_device("correction", gx.data_ptr(), to_engine=False,
                                       as_double=gx.dtype == torch.float64,
                                       stream=torch.cuda.current_stream(x.device).cuda_stream)
        gx = gx.to(x.dtype) * g
        gb = torch.as_tensor(terms[:, 1] * g, dtype=background.dtype, device=background.device)
        gp = torch.as_tensor((terms[:, 1] - terms[:, 2]) * g, dtype=pedestal.dtype, device=pedestal.device)
        gpsf = None
        if ctx.has_psf:
            out = np.zeros(ps.shape, np.float64)
            for k in range(model.nexp):
                gn = model.engine.psf_gradient(k, ps[k].shape)      # dL/d(psf_k / sum psf_k)
                s = ps[k].sum()
                psi = ps[k] / s
                out[k] = (gn - float((gn * psi).sum())) / s          # through the normalisation
            gpsf = torch.as_tensor(out * g, dtype=psf.dtype, device=psf.device)
        return gx, gb, gp, gpsf, None
