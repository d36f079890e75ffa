"""Differentiable list-mode strip projection for PyTorch.

    y = project(rec, rho, sigma)        y_e = sum_j K_ej(sigma) rho_j  (x s_j in MODE_GPU)

over the events held by ``rec`` (a stripmlem.Reconstruction), with the pixel
set of every event fixed by the geometry's sigmas.  Backward runs the
library's adjoint kernel for d/drho (g_j = sum_e w_e K_ej) and its sigma
kernel for d/d(sigma_z, sigma_dl) (GaussianKernel, MODE_CPU).  All three are
hand-written sm_100a kernels called through the C ABI on device buffers
(strip_forward_device / strip_adjoint_device / strip_grad_sigma_device).

fit_sigma() fits (sigma_z, sigma_dl) by maximising the extended list-mode
Poisson likelihood of the events for a known activity image:

    l(sigma) = sum_e log y_e(sigma) - N log Lambda(sigma),
    Lambda(sigma) = sum_c v_c y_c(sigma)

where the normalisation Lambda integrates the model over the event space by
quadrature: y_c is the projection of a regular grid of quadrature events c
(cell volume v_c) held by a second context.  The reference has no model fit;
its kernels are GaussianKernel (src/2d/strip/gaussian_kernel.h:27-160) and
AnalyticKernel (src/2d/strip/analytic_kernel.h:28-62).
"""
import math

import numpy as np
import torch

from . import MODE_CPU, Reconstruction, StripError, _lib


def _sync(t):
    if t.is_cuda:
        torch.cuda.current_stream(t.device).synchronize()


def _check_rho(rec, rho):
    n_y, n_z = rec.scanner.n_y_pixels, rec.scanner.n_z_pixels
    if rho.numel() != n_y * n_z:
        raise ValueError(f"rho must hold {n_y} x {n_z} values")
    if not rho.is_cuda or rho.device.index != rec.device:
        raise ValueError(f"rho must live on {rec.torch_device}")


def _sigmas(sigma):
    s = sigma.detach().to("cpu", torch.float64)
    return float(s[0]), float(s[1])


class StripProjection(torch.autograd.Function):
    """y = P(sigma) rho for the events of a context (see module docstring)."""

    @staticmethod
    def forward(ctx, rho, sigma, rec, mode):
        _check_rho(rec, rho)
        sz, sdl = _sigmas(sigma)
        img = rho.detach().to(torch.float32).contiguous()
        y = torch.empty(rec.n_events, dtype=torch.float64, device=rho.device)
        _sync(img)
        rec._check(rec.lib.strip_forward_device(rec._ctx, img.data_ptr(), sz, sdl,
                                                int(mode), y.data_ptr()))
        ctx.save_for_backward(img, sigma)
        ctx.rec = rec
        ctx.mode = int(mode)
        ctx.rho_shape = rho.shape
        ctx.rho_dtype = rho.dtype
        return y

    @staticmethod
    def backward(ctx, gy):
        img, sigma = ctx.saved_tensors
        rec, mode = ctx.rec, ctx.mode
        sz, sdl = _sigmas(sigma)
        w = gy.detach().to(device=img.device, dtype=torch.float64).contiguous()
        _sync(w)
        g_rho = g_sigma = None
        if ctx.needs_input_grad[0]:
            g = torch.empty(img.numel(), dtype=torch.float64, device=img.device)
            rec._check(rec.lib.strip_adjoint_device(rec._ctx, w.data_ptr(), sz, sdl, mode,
                                                    g.data_ptr()))
            g_rho = g.reshape(ctx.rho_shape).to(ctx.rho_dtype)
        if ctx.needs_input_grad[1]:
            if mode != MODE_CPU:
                raise StripError(_lib.STRIP_E_INVALID,
                                 "the sigma gradient is defined for the GaussianKernel "
                                 "(MODE_CPU)")
            out = torch.empty(2, dtype=torch.float64, device=img.device)
            rec._check(rec.lib.strip_grad_sigma_device(rec._ctx, img.data_ptr(), w.data_ptr(),
                                                       sz, sdl, out.data_ptr()))
            g_sigma = out.to(device=sigma.device, dtype=sigma.dtype)
        return g_rho, g_sigma, None, None


def project(rec, rho, sigma=None, mode=None):
    """Differentiable forward projection of ``rho`` (CUDA tensor, n_y x n_z,
    on the context's device) with kernel sigmas ``sigma`` (tensor [sigma_z,
    sigma_dl]; default the geometry's) over the events of ``rec``; returns
    the float64 per-event intensities in the caller's event order."""
    if sigma is None:
        sigma = torch.tensor([rec.scanner.sigma_z, rec.scanner.sigma_dl],
                             dtype=torch.float64)
    return StripProjection.apply(rho, sigma, rec, rec.mode if mode is None else mode)


def quadrature_events(scanner, h_z, h_dl, margin_dl=None):
    """Midpoints of a regular grid over the detected event space
    |z_u|, |z_d| < L/2 and |dl| up to the largest strip separation plus a
    margin (default 6 sigma_dl); returns (z_u, z_d, dl, cell_volume)."""
    R, L = scanner.radius, scanner.scintillator_length
    if margin_dl is None:
        margin_dl = 6.0 * scanner.sigma_dl
    dmax = 2.0 * R * math.sqrt(1.0 + (L / (2.0 * R)) ** 2) + margin_dl
    nz = max(1, int(round(L / h_z)))
    nd = max(1, int(math.ceil(2.0 * dmax / h_dl)))
    hz = L / nz
    gz = -L / 2 + hz * (np.arange(nz) + 0.5)
    gd = -nd * h_dl / 2 + h_dl * (np.arange(nd) + 0.5)
    a, b, c = np.meshgrid(gz, gz, gd, indexing="ij")
    return (a.ravel().astype(np.float32), b.ravel().astype(np.float32),
            c.ravel().astype(np.float32), hz * hz * h_dl)


def log_likelihood(rec_data, rec_norm, cell_volume, rho, sigma, weights=None):
    """Extended list-mode log-likelihood l(sigma) (module docstring); events
    whose projection is zero (empty pixel set) do not count.  ``weights``
    (float64 tensor, one per event of rec_data) weighs the events."""
    y = project(rec_data, rho, sigma, MODE_CPU)
    yq = project(rec_norm, rho, sigma, MODE_CPU)
    pos = y > 0
    if weights is None:
        data = torch.log(y[pos]).sum()
        n = pos.sum()
    else:
        w = weights[pos]
        data = (w * torch.log(y[pos])).sum()
        n = w.sum()
    return data - n * torch.log(cell_volume * yq.sum())


def fit_sigma(rec_data, rec_norm, cell_volume, rho, sigma0, max_iter=60,
              weights=None, callback=None):
    """Fits (sigma_z, sigma_dl) from sigma0, maximising log_likelihood() by
    L-BFGS with a strong-Wolfe line search on log sigma (two parameters, a
    smooth objective).  Returns (sigma, history of (l, sigma_z, sigma_dl) per
    objective evaluation).  rec_data holds the events, rec_norm the
    quadrature events."""
    logs = torch.tensor([math.log(sigma0[0]), math.log(sigma0[1])], dtype=torch.float64,
                        requires_grad=True)
    opt = torch.optim.LBFGS([logs], lr=1.0, max_iter=max_iter, tolerance_grad=1e-9,
                            tolerance_change=1e-12, history_size=10,
                            line_search_fn="strong_wolfe")
    scale = 1.0 / max(1, rec_data.n_events)
    hist = []

    def closure():
        opt.zero_grad()
        sigma = torch.exp(logs)
        ll = log_likelihood(rec_data, rec_norm, cell_volume, rho, sigma, weights)
        loss = -ll * scale
        loss.backward()
        s = sigma.detach()
        hist.append((float(ll.detach()), float(s[0]), float(s[1])))
        if callback is not None:
            callback(len(hist) - 1, hist[-1])
        return loss

    opt.step(closure)
    return torch.exp(logs).detach(), hist


__all__ = ["StripProjection", "project", "quadrature_events", "log_likelihood",
           "fit_sigma", "Reconstruction"]
