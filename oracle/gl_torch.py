"""Differentiable FP64 restatement of the oracle's eta path, for gradients.

TEST INFRASTRUCTURE ONLY.  A line-by-line torch transliteration of
``oracle/gl_oracle.py``'s ``first_order``, ``eta22`` and the eta half of
``order3`` (which restate ``python/src/green_laplace/spatial.py:74-79,
156-231`` and ``_order3.py:18-148, 175-287``), evaluated with
``torch.fft`` in complex128 on the CPU so that ``torch.autograd`` gives the
reference gradient of a loss of ``eta11 + eta22 + eta33`` with respect to the
first-order amplitudes.  The reference has no gradient of its own, so the
gradient parity of the engine is pinned by this autograd reference and by
central finite differences of ``oracle/gl_oracle.py`` (tests check that the
two agree).

Supports, shifts, scales, the peak and the roundoff-floor decisions are
computed from detached values exactly as the oracle computes them: the
derivative is that of the map on its current piece, which is what the
engine's adjoint computes.
"""

from __future__ import annotations

import numpy as np
import torch

from . import gl_oracle as O


def _t(x: np.ndarray) -> torch.Tensor:
    return torch.as_tensor(np.asarray(x))


def _floor(h: torch.Tensor, support: np.ndarray) -> torch.Tensor:
    """``zero_below_roundoff_floor`` (``_spectral.py:52-64``) with the kept
    bins chosen on detached values."""
    mags = h.detach().abs().numpy()
    if not np.any(support):
        return h
    peak = float(np.max(mags[support]))
    if peak == 0.0:
        return h
    floor = 16.0 * O.EPS * max(1.0, np.log2(h.numel()))
    zero = support & (mags < floor * peak)
    return torch.where(_t(zero), torch.zeros_like(h), h)


def _mask(h: torch.Tensor, support: np.ndarray) -> torch.Tensor:
    return torch.where(_t(support), h, torch.zeros_like(h))


def deposit(a: torch.Tensor, b: torch.Tensor, kx, ky, omega, depth, lx, ly, nx, ny, t):
    """``deposit_modes`` (``src/gl_spectral_surface.m:123-149``) as a torch op."""
    mx = O.matlab_round(np.asarray(kx) / (2.0 * np.pi / lx)).astype(np.int64)
    my = O.matlab_round(np.asarray(ky) / (2.0 * np.pi / ly)).astype(np.int64)
    flat = torch.as_tensor((my % ny) * nx + (mx % nx))
    phase = torch.as_tensor(np.exp(-1j * np.asarray(omega) * t))
    vals = float(nx * ny) * torch.complex(a / depth, b / depth) * phase
    s = torch.zeros(ny * nx, dtype=torch.complex128)
    s = s.index_add(0, flat, vals)
    return s.reshape(ny, nx)


def eta22(s: torch.Tensor, qx, qy, rank: int) -> torch.Tensor:
    """``gl_oracle.eta22`` (``spatial.py:156-231``): the analytic eta22/h."""
    g = O.Geometry(qx, qy)
    sn = s.detach().numpy()
    support = O.support_of(sn)
    out_support = O.minkowski_support(support, 2)
    qp = O.peak_q_of(sn, support, g.q)
    lam = np.sqrt((2.0 * np.sqrt(qp * np.tanh(qp))) ** 2 - 2.0 * qp * np.tanh(2.0 * qp))
    nodes, weights = O.gauss_laguerre(rank)
    shift = 0.5 * (float(np.min(g.nu[support])) + float(np.max(g.sqrt_a[out_support])) / 2.0)
    q2 = g.q**2
    banks = (None, g.nu, g.nu**2, g.qx / g.safe_nu, g.qy / g.safe_nu, q2 / g.safe_nu, g.qx, g.qy)
    acc = torch.zeros_like(s)
    for x, w in zip(nodes, weights):
        tau = x / lam
        damped = s * _t(np.exp(-tau * (g.nu - shift)))
        v, v_nu, v_nu2, hx, hy, rad, jx, jy = (
            torch.fft.ifft2(damped if m is None else damped * _t(m)) for m in banks)
        sd = 2.0 * v * v_nu2 + v_nu**2 - hx**2 - hy**2
        sk = 2.0 * v * rad + 2.0 * (hx * jx + hy * jy)
        coef = w * np.exp(x) / lam / 4.0 * np.exp(-2.0 * shift * tau)
        sh = O.sinh_over_root(g.sqrt_a, tau)
        sd_hat = _floor(_mask(torch.fft.fft2(sd), out_support), out_support)
        sk_hat = _floor(_mask(torch.fft.fft2(sk), out_support), out_support)
        acc = acc + coef * (_t(-g.a * sh) * sd_hat + _t(np.cosh(g.sqrt_a * tau)) * sk_hat)
    return torch.fft.ifft2(acc)


def eta33(s: torch.Tensor, qx, qy, *, inner_rank: int = 4, outer_rank: int = 4) -> torch.Tensor:
    """The eta half of ``gl_oracle.order3`` (``_order3.py:18-148``): eta33/h."""
    g = O.Geometry(qx, qy)
    sn = s.detach().numpy()
    support = O.support_of(sn)
    hat = np.fft.fft2(support.astype(float))
    s2 = np.real(np.fft.ifft2(hat**2)) > 0.5
    s3 = np.real(np.fft.ifft2(hat**3)) > 0.5
    nu_min = float(np.min(g.nu[support]))
    shift2 = 0.5 * (nu_min + float(np.max(g.sqrt_a[s2])) / 2.0)
    shift3 = 0.5 * (nu_min + float(np.max(g.sqrt_a[s3])) / 3.0)
    qp = O.peak_q_of(sn, support, g.q)
    peak_nu = np.sqrt(qp * np.tanh(qp))
    lam2 = 2.0 * peak_nu - np.sqrt(2.0 * qp * np.tanh(2.0 * qp))
    lam3 = 3.0 * peak_nu - np.sqrt(3.0 * qp * np.tanh(3.0 * qp))
    inodes, iweights = O.gauss_laguerre(inner_rank)
    onodes, oweights = O.gauss_laguerre(outer_rank)
    q2 = g.q**2
    first_bank = (None, 1j * g.qx, 1j * g.qy, g.qx / g.safe_nu, g.qy / g.safe_nu, -1j * g.nu,
                  g.nu * g.qx, g.nu * g.qy, -1j * q2 / g.safe_nu, -1j * q2 * g.nu, -g.a, -q2)
    first_names = ("eta", "etax", "etay", "phix", "phiy", "phiz", "phixz", "phiyz", "phizz",
                   "phizzz", "phitz", "phitzz")
    inner_bank = (None, g.nu, g.nu**2, g.nu**3, g.qx / g.safe_nu, g.qy / g.safe_nu, g.qx, g.qy,
                  q2 / g.safe_nu, q2, g.nu * g.qx, g.nu * g.qy)
    dx, dy = _t(1j * g.qx), _t(1j * g.qy)
    eta_hat = torch.zeros_like(s)
    for x, w in zip(onodes, oweights):
        tau = x / lam3
        damped = s * _t(np.exp(-tau * (g.nu - shift3)))
        f = {k: torch.fft.ifft2(damped if m is None else _t(m) * damped)
             for k, m in zip(first_names, first_bank)}
        e_hat = torch.zeros_like(s)
        p_hat = torch.zeros_like(s)
        pt_hat = torch.zeros_like(s)
        for xi, wi in zip(inodes, iweights):
            t2 = xi / lam2
            d2 = damped * _t(np.exp(-t2 * (g.nu - shift2)))
            v, v1, v2, v3, hx, hy, jx, jy, rad, qq, njx, njy = (
                torch.fft.ifft2(d2 if m is None else d2 * _t(m)) for m in inner_bank)
            sources = (
                2.0 * v * v2 + v1**2 - hx**2 - hy**2,
                2.0 * v * rad + 2.0 * (hx * jx + hy * jy),
                2.0 * v * v3 + 4.0 * v1 * v2 - 2.0 * hx * jx - 2.0 * hy * jy,
                2.0 * (v1 * rad + v * qq) + 2.0 * (jx**2 + hx * njx + jy**2 + hy * njy),
            )
            sd, sk, sdt, skt = (_floor(_mask(torch.fft.fft2(src), s2), s2) for src in sources)
            sh = _t(O.sinh_over_root(g.sqrt_a, t2))
            ch = _t(np.cosh(g.sqrt_a * t2))
            coef = wi * np.exp(xi) / lam2 * np.exp(-2.0 * shift2 * t2) / 4.0
            e_hat = e_hat + coef * (_t(-g.a) * sh * sd + ch * sk)
            p_hat = p_hat + 1j * coef * (ch * sd - sh * sk)
            pt_hat = pt_hat + coef * (ch * sdt - sh * skt)
        e_hat, p_hat, pt_hat = (_mask(h, s2) for h in (e_hat, p_hat, pt_hat))
        pair = {
            "eta": torch.fft.ifft2(e_hat),
            "etax": torch.fft.ifft2(dx * e_hat),
            "etay": torch.fft.ifft2(dy * e_hat),
            "phix": torch.fft.ifft2(dx * p_hat),
            "phiy": torch.fft.ifft2(dy * p_hat),
            "phiz": torch.fft.ifft2(_t(g.a) * p_hat),
            "phizz": torch.fft.ifft2(_t(q2) * p_hat),
            "phitz": torch.fft.ifft2(_t(g.a) * pt_hat),
        }
        fe, p = f["eta"], pair
        k_pair = (f["phix"] * p["etax"] + f["phiy"] * p["etay"] + p["phix"] * f["etax"]
                  + p["phiy"] * f["etay"] - fe * p["phizz"] - p["eta"] * f["phizz"])
        k_direct = fe * (f["phixz"] * f["etax"] + f["phiyz"] * f["etay"]) - 0.5 * fe**2 * f["phizzz"]
        d_pair = (fe * p["phitz"] + p["eta"] * f["phitz"] + f["phix"] * p["phix"]
                  + f["phiy"] * p["phiy"] + f["phiz"] * p["phiz"])
        d_direct = (0.5 * fe**2 * f["phitzz"]
                    + fe * (f["phix"] * f["phixz"] + f["phiy"] * f["phiyz"] + f["phiz"] * f["phizz"]))
        fk = k_direct / 4.0 + k_pair / 2.0
        fd = d_direct / 4.0 + d_pair / 2.0
        fk_hat = _floor(_mask(torch.fft.fft2(fk), s3), s3)
        fd_hat = _floor(_mask(torch.fft.fft2(fd), s3), s3)
        sh = _t(O.sinh_over_root(g.sqrt_a, tau))
        ch = _t(np.cosh(g.sqrt_a * tau))
        coef = w * np.exp(x) / lam3 * np.exp(-3.0 * shift3 * tau)
        eta_hat = eta_hat + coef * (_t(g.a) * sh * fd_hat - 1j * ch * fk_hat)
    return torch.fft.ifft2(_mask(eta_hat, s3))


def eta_surface(a: torch.Tensor, b: torch.Tensor, *, kx, ky, omega, depth, lx, ly, nx, ny, t,
                components=("eta11", "eta22", "eta33"), eta22_rank: int = 6,
                inner_rank: int = 4, outer_rank: int = 4) -> torch.Tensor:
    """Physical surface h Re(sum of the analytic components) for one snapshot."""
    kxg, kyg = O.fft_wavenumber_grid(lx, ly, nx, ny)
    qx, qy = depth * kxg, depth * kyg
    s = deposit(a, b, kx, ky, omega, depth, lx, ly, nx, ny, t)
    total = torch.zeros_like(s)
    if "eta11" in components:
        total = total + torch.fft.ifft2(s)
    if "eta22" in components:
        total = total + eta22(s, qx, qy, eta22_rank)
    if "eta33" in components:
        total = total + eta33(s, qx, qy, inner_rank=inner_rank, outer_rank=outer_rank)
    return depth * total.real
