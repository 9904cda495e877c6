"""The differentiable model (updc_b200/autograd.py, nll.cuh).

CPU: the oracle's H^T (the reference's scatter + frequency-domain adjoint,
updc_core.c:988-995, 1175-1176, 1280-1287) is the adjoint of its forward
model S P, checked with random vectors.

GPU: gradients of the weighted Poisson NLL with respect to x, per-exposure
background and pedestal and the Gaussian-core PSF width, against FP64
central finite differences (relative step 1e-6) and, for x, against the
reference's H^T applied to W (ratio - 1) through the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import fft_shape_for


def _solver(oracle, ds, precision):
    w = ds.workload
    fw, fh = fft_shape_for(ds)
    return oracle.Solver(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=precision)


def _gather(oracle, ds, blur_k, k):
    """S_k applied to a target plane (detector values; pixels without links are 0)."""
    w = ds.workload
    off, tgt, frac, _ = oracle.linkmap_decode(str(ds.rows[k].links), w.iw, w.ih, w.W, w.H)
    pix = np.repeat(np.arange(w.iw * w.ih), np.diff(off.astype(np.int64)))
    out = np.zeros(w.iw * w.ih)
    np.add.at(out, pix, frac.astype(np.float64) * blur_k.reshape(-1).astype(np.float64)[tgt])
    return out.reshape(w.ih, w.iw)


def test_oracle_adjoint_is_the_transpose_of_the_forward_model(oracle, datasets):
    ds = datasets("small")
    w = ds.workload
    s = _solver(oracle, ds, 64)
    rng = np.random.default_rng(11)
    u = rng.standard_normal((w.H, w.W))
    v = rng.standard_normal((w.nexp, w.ih, w.iw))
    s.estimate[...] = u
    hu = np.stack([_gather(oracle, ds, s.forward_blur(k), k) for k in range(w.nexp)])
    htv = s.adjoint(v)
    lhs = float(np.sum(hu * v))
    rhs = float(np.sum(u * htv))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0), (lhs, rhs)


# ---------------------------------------------------------------------------- GPU
def _model(ds, form):
    from updc_b200.autograd import PoissonModel
    w = ds.workload
    return PoissonModel(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, form=form)


def _inputs(model, ds, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    w = ds.workload
    x0 = model.engine.plane("estimate", as_double=True)
    x0 = np.maximum(x0, 0.0) + 0.05                       # positive, so every mu > 0
    bkg = torch.tensor(rng.uniform(0.1, 1.0, w.nexp), dtype=torch.float64)
    ped = torch.tensor(rng.uniform(5.0, 20.0, w.nexp), dtype=torch.float64)
    return x0, bkg, ped


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("form,tol", [("fp64", 1e-10), ("fp32", 2e-5)])
def test_x_gradient_matches_reference_adjoint(engine_lib, oracle, datasets, form, tol):
    """dL/dx = H^T (W (1 - ratio)) against the reference's H^T of the same residual."""
    import torch
    ds = datasets("medium")
    model = _model(ds, form)
    x0, bkg, ped = _inputs(model, ds)
    x = torch.tensor(x0, dtype=model.dtype, device="cuda", requires_grad=True)
    loss = model.loss(x, bkg, ped)
    loss.backward()
    r = np.stack([model.engine.plane("wr", k, as_double=True) for k in range(ds.workload.nexp)])
    s = _solver(oracle, ds, 64)
    ref = s.adjoint(r)                   # reference H^T applied to W (1 - ratio) = -W (ratio - 1)
    assert _rel(x.grad.double().cpu().numpy(), ref) <= tol
    model.close()


@pytest.mark.gpu
def test_gradients_match_fp64_finite_differences(engine_lib, oracle, datasets):
    """x (256 random pixels), background, pedestal and PSF sigma against FP64
    central differences with a relative step of 1e-6; both the FP64 and the
    FP32 analytic gradients are checked."""
    import torch
    from updc_b200.autograd import gauss_moffat_psf
    ds = datasets("medium")
    w = ds.workload
    m64 = _model(ds, "fp64")
    m32 = _model(ds, "fp32")
    x0, bkg, ped = _inputs(m64, ds)
    psize = ds.rows[0].psf_width
    sigma0 = 1.2

    def psfs(sig):
        p = gauss_moffat_psf(psize, sig)
        return p.unsqueeze(0).expand(w.nexp, psize, psize)

    def analytic(model):
        x = torch.tensor(x0, dtype=model.dtype, device="cuda", requires_grad=True)
        b = bkg.clone().requires_grad_(True)
        p = ped.clone().requires_grad_(True)
        sig = torch.tensor(sigma0, dtype=torch.float64, requires_grad=True)
        loss = model.loss(x, b, p, psfs(sig))
        loss.backward()
        return (x.grad.double().cpu().numpy(), b.grad.numpy().copy(), p.grad.numpy().copy(), float(sig.grad))

    g64 = analytic(m64)
    g32 = analytic(m32)

    def parts64(x=None, b=None, p=None, sig=sigma0):
        # per-block partial sums of L: differences taken partial by partial
        # are exact where nothing changed
        xt = torch.tensor(x0 if x is None else x, dtype=torch.float64, device="cuda")
        m64._load(xt, bkg if b is None else b, ped if p is None else p, psfs(sig))
        m64.engine.nll()
        return m64.engine.nll_partials()[..., 0]

    def fd(plus, minus, h):
        return float(np.sum(plus - minus)) / (2 * h)

    # x: the forward model is linear in x, so mu(x0 +- h e_p) = mu0 +- h S P e_p
    # exactly; the central difference is evaluated on the detector pixels the
    # step reaches, from the FP64 model's blur planes, with
    # l(mu + d) - l(mu - d) = W (2 d - y log1p(2 d / (mu - d))), which keeps
    # single-pixel steps of 1e-6 relative exact to ~1e-12 (re-running the
    # FFT forward model for each step would bury them in its rounding noise)
    parts64()                                        # FP64 forward planes at x0, bkg, ped, sigma0
    blur = [m64.engine.plane("blur", k, as_double=True) for k in range(w.nexp)]
    wht = [m64.engine.plane("weight", k, as_double=True).ravel() for k in range(w.nexp)]
    sci = [m64.engine.plane("science", k, as_double=True).ravel() for k in range(w.nexp)]
    psi = psfs(sigma0)[0].numpy()
    psi = psi / psi.sum()
    ph_, pw_ = psi.shape
    cy, cx = ph_ // 2, pw_ // 2
    maps = []
    for k in range(w.nexp):
        off, tgt, frac, _ = oracle.linkmap_decode(str(ds.rows[k].links), w.iw, w.ih, w.W, w.H)
        off = off.astype(np.int64)
        tgt = tgt.astype(np.int64)
        pix = np.repeat(np.arange(w.iw * w.ih), np.diff(off))
        order = np.argsort(tgt, kind="stable")
        maps.append((off, tgt, frac.astype(np.float64), tgt[order], pix[order]))

    def fd_pixel(py, px, h):
        total = 0.0
        ys = np.arange(max(0, py - cy), min(w.H, py - cy + ph_))
        xs = np.arange(max(0, px - cx), min(w.W, px - cx + pw_))
        dplane = np.zeros((w.H, w.W))
        dplane[np.ix_(ys, xs)] = psi[np.ix_(ys - py + cy, xs - px + cx)]
        foot = (ys[:, None] * w.W + xs[None, :]).ravel()
        for k in range(w.nexp):
            off, tgt, frac, tsort, psort = maps[k]
            lo = np.searchsorted(tsort, foot, "left")
            hi = np.searchsorted(tsort, foot, "right")
            n2 = hi - lo
            seg2 = np.concatenate([[0], np.cumsum(n2)[:-1]])
            dets = np.unique(psort[np.repeat(lo - seg2, n2) + np.arange(int(n2.sum()))])
            dets = dets[wht[k][dets] > 0]
            if dets.size == 0:
                continue
            starts, lens = off[dets], off[dets + 1] - off[dets]
            seg = np.concatenate([[0], np.cumsum(lens)[:-1]])
            idx = np.repeat(starts - seg, lens) + np.arange(int(lens.sum()))
            mu0 = np.add.reduceat(frac[idx] * blur[k].ravel()[tgt[idx]], seg) + float(bkg[k]) + float(ped[k])
            dmu = np.add.reduceat(frac[idx] * dplane.ravel()[tgt[idx]], seg)
            y = sci[k][dets] + float(ped[k])
            d = h * dmu
            total += float(np.sum(wht[k][dets] * (2.0 * d - y * np.log1p(2.0 * d / (mu0 - d)))))
        return total / (2.0 * h)

    rng = np.random.default_rng(5)
    flat = rng.choice(w.W * w.H, 256, replace=False)
    fd_x, an64, an32 = [], [], []
    for t in flat:
        yy, xx = divmod(int(t), w.W)
        fd_x.append(fd_pixel(yy, xx, 1e-6 * abs(x0[yy, xx])))
        an64.append(g64[0][yy, xx])
        an32.append(g32[0][yy, xx])
    fd_x, an64, an32 = map(np.array, (fd_x, an64, an32))
    scale = np.sqrt(np.mean(an64 ** 2))
    err64 = np.max(np.abs(an64 - fd_x)) / scale
    err32 = np.max(np.abs(an32 - fd_x)) / scale
    print(f"x: FD vs FP64 analytic {err64:.2e}, vs FP32 analytic {err32:.2e} (of the gradient's RMS)")
    assert err64 <= 1e-8 and err32 <= 1e-4, (err64, err32)

    for which, base, g_an64, g_an32 in (("b", bkg, g64[1], g32[1]), ("p", ped, g64[2], g32[2])):
        for k in range(w.nexp):
            h = 1e-6 * abs(float(base[k]))
            up, dn = base.clone(), base.clone()
            up[k] += h
            dn[k] -= h
            f = fd(parts64(**{which: up}), parts64(**{which: dn}), h)
            assert abs(g_an64[k] - f) <= 1e-5 * abs(f), (which, k, g_an64[k], f)
            assert abs(g_an32[k] - f) <= 1e-4 * abs(f), (which, k, g_an32[k], f)

    h = 1e-6 * sigma0
    f = fd(parts64(sig=sigma0 + h), parts64(sig=sigma0 - h), h)
    print(f"sigma: FD {f:.9g}, FP64 analytic {g64[3]:.9g}, FP32 analytic {g32[3]:.9g}")
    assert abs(g64[3] - f) <= 1e-5 * abs(f), (g64[3], f)
    assert abs(g32[3] - f) <= 1e-4 * abs(f), (g32[3], f)
    m64.close()
    m32.close()


@pytest.mark.gpu
def test_backward_recomputes_from_inputs(engine_lib, datasets):
    """Two forward calls before one backward: the backward uses its own
    saved inputs (the engine's planes are workspace, not saved state)."""
    import torch
    ds = datasets("c0")
    model = _model(ds, "fp64")
    x0, bkg, ped = _inputs(model, ds)
    xa = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    la = model.loss(xa, bkg, ped)
    la.backward()
    ga = xa.grad.clone()
    xa.grad = None
    la2 = model.loss(xa, bkg, ped)
    xb = torch.tensor(2.0 * x0, dtype=torch.float64, device="cuda", requires_grad=True)
    _ = model.loss(xb, bkg, ped)          # overwrites the engine's planes
    la2.backward()
    assert torch.equal(xa.grad, ga)
    model.close()
