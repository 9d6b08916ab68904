"""CPU oracle for the Green--Laplace (GL) spatial bound-wave path.

TEST INFRASTRUCTURE ONLY.  This module is a plain FP64 NumPy restatement of
the reference algorithm (Xinyu01091002/green-laplace-wave-reconstruction
v0.5.0).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg may import it, and only as the checker or the timed CPU baseline.
The product path (``gl_engine``) never calls into this module.

Parity pin: the functions below are checked against the reference's own
MATLAB-generated golden fields (``python/tests/fixtures/*.json``, copied into
``tests/golden/matlab_fixtures.npz``) and against outputs of the reference
Python package generated by ``tests/golden/make_golden.py``.

Every function names the reference file:line it restates.  Array layout is
the reference's: ``[iy, ix]`` (row = y, column = x), FFT bin order as
``numpy.fft.fftfreq``; spectra are N^2-scaled (``fft2`` convention).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

EPS = float(np.finfo(float).eps)
TINY = float(np.finfo(float).tiny)

# ---------------------------------------------------------------------------
# grid, support and roundoff helpers
# ---------------------------------------------------------------------------


def fft_wavenumber_grid(lx: float, ly: float, nx: int, ny: int):
    """kx, ky meshgrids (``python/src/green_laplace/_spectral.py:9-16``)."""
    if lx <= 0 or ly <= 0 or nx < 2 or ny < 2 or nx % 2 or ny % 2:
        raise ValueError("positive domain lengths and positive even grid sizes are required")
    kx_line = 2.0 * np.pi * np.fft.fftfreq(nx, d=lx / nx)
    ky_line = 2.0 * np.pi * np.fft.fftfreq(ny, d=ly / ny)
    return np.meshgrid(kx_line, ky_line)


def mode_index_grid(nx: int, ny: int):
    """Signed integer mode numbers (mx, my) per bin, fftfreq order."""
    mx_line = np.rint(np.fft.fftfreq(nx) * nx).astype(np.int64)
    my_line = np.rint(np.fft.fftfreq(ny) * ny).astype(np.int64)
    return np.meshgrid(mx_line, my_line)


def support_of(spectrum: np.ndarray) -> np.ndarray:
    """Parent support |s| > 1e-13 max(1, max|s|) (``spatial.py:163-164``, ``_order3.py:33-34``)."""
    threshold = 1.0e-13 * max(1.0, float(np.max(np.abs(spectrum))))
    return np.abs(spectrum) > threshold


def minkowski_support(indicator: np.ndarray, power: int) -> np.ndarray:
    """``ifft2(fft2(1_S)^power) > 0.5`` (``_order3.py:38-40``, ``spatial.py:169-170``)."""
    transform = np.fft.fft2(indicator.astype(float))
    return np.real(np.fft.ifft2(transform**power)) > 0.5


def zero_below_roundoff_floor(spectrum: np.ndarray, support: np.ndarray) -> np.ndarray:
    """Source-local FFT roundoff suppression (``_spectral.py:52-64``).

    Bins of ``support`` whose modulus is below
    ``16 eps max(1, log2(size)) max_support|x|`` are set to zero.
    """
    out = spectrum.copy()
    magnitudes = np.abs(out[support])
    if magnitudes.size == 0:
        return out
    peak = float(np.max(magnitudes))
    if peak == 0.0:
        return out
    floor = 16.0 * EPS * max(1.0, np.log2(out.size))
    out[support & (np.abs(out) < floor * peak)] = 0.0
    return out


def check_alias_safe(support: np.ndarray, order: int) -> None:
    """Nyquist guards (``_spectral.py:67-77`` for order 2, ``_order3.py:290-296`` for 3)."""
    ny, nx = support.shape
    if not np.any(support):
        raise ValueError("eta1 has empty analytic support")
    mx, my = mode_index_grid(nx, ny)
    if np.max(order * np.abs(mx[support])) >= nx / 2.0 or np.max(
        order * np.abs(my[support])
    ) >= ny / 2.0:
        if order == 2:
            raise ValueError("quadratic output support reaches a Nyquist boundary")
        raise ValueError("cubic output support reaches a Nyquist boundary")


def gauss_laguerre(rank: int):
    """Golub--Welsch Gauss--Laguerre rule with moment gate (``quadrature.py:11-31``)."""
    if not isinstance(rank, int) or rank < 1:
        raise ValueError("rank must be a positive integer")
    jacobi = np.diag(2.0 * np.arange(1, rank + 1) - 1.0)
    if rank > 1:
        off = np.arange(1, rank, dtype=float)
        jacobi += np.diag(off, 1) + np.diag(off, -1)
    nodes, vectors = np.linalg.eigh(jacobi)
    weights = vectors[0, :] ** 2
    for degree in range(2 * rank):
        exact = math.factorial(degree)
        if abs(np.sum(weights * nodes**degree) - exact) / max(1, exact) > 3.0e-11:
            raise ArithmeticError(
                f"Gauss--Laguerre moment check failed at rank={rank}, degree={degree}"
            )
    return nodes, weights


def dispersion_q(omega, depth: float, gravity: float = 9.81) -> np.ndarray:
    """Newton solve of q tanh q = omega^2 h/g (``dispersion.py:19-42``)."""
    values = np.asarray(omega, dtype=float)
    if depth <= 0 or gravity <= 0 or np.any(values < 0):
        raise ValueError("depth and gravity must be positive and omega nonnegative")
    target = values**2 * depth / gravity
    q = np.maximum(np.where(target < 1.0, np.sqrt(target), target), TINY)
    for _ in range(40):
        th = np.tanh(q)
        step = (q * th - target) / np.maximum(th + q * (1.0 - th**2), TINY)
        cand = np.maximum(q - step, 0.5 * q)
        done = np.max(np.abs(cand - q) / np.maximum(1.0, q)) < 5.0e-15
        q = cand
        if done:
            break
    if not np.allclose(q * np.tanh(q), target, rtol=2.0e-13, atol=2.0e-15):
        raise ArithmeticError("finite-depth dispersion solve did not converge")
    return q


def sinh_over_root(sqrt_a: np.ndarray, tau: float) -> np.ndarray:
    """sinh(sqrt(A) tau)/sqrt(A), with the tau limit at A=0 (``_order3.py:124-126``)."""
    out = np.full_like(sqrt_a, tau)
    nz = sqrt_a > 0
    out[nz] = np.sinh(sqrt_a[nz] * tau) / sqrt_a[nz]
    return out


@dataclass
class Geometry:
    """Dimensionless per-bin tables shared by the executors."""

    qx: np.ndarray
    qy: np.ndarray
    q: np.ndarray = field(init=False)
    nu: np.ndarray = field(init=False)
    a: np.ndarray = field(init=False)
    sqrt_a: np.ndarray = field(init=False)
    safe_nu: np.ndarray = field(init=False)

    def __post_init__(self):
        self.q = np.hypot(self.qx, self.qy)
        self.a = self.q * np.tanh(self.q)
        self.nu = np.sqrt(self.q * np.tanh(self.q))
        self.sqrt_a = np.sqrt(self.a)
        self.safe_nu = np.maximum(self.nu, TINY)


def peak_q_of(spectrum: np.ndarray, support: np.ndarray, q: np.ndarray) -> float:
    """Peak wavenumber: first argmax of |s|^2 over the support (``spatial.py:176-178``)."""
    amplitudes = np.abs(spectrum[support]) ** 2
    flat = np.flatnonzero(support)[int(np.argmax(amplitudes))]
    return float(q.flat[flat])


# ---------------------------------------------------------------------------
# order two
# ---------------------------------------------------------------------------

# eta22 / psi22 multiplier banks (``spatial.py:196-203, 405-413``); each
# applies its factors in the reference's left-to-right order, e.g.
# ``(damped * qx) / safe_nu``.
def _eta22_banks(g: Geometry):
    q2 = g.q**2
    return (
        lambda d: d,  # v
        lambda d: d * g.nu,  # v_nu
        lambda d: d * g.nu**2,  # v_nu2
        lambda d: d * g.qx / g.safe_nu,  # hx
        lambda d: d * g.qy / g.safe_nu,  # hy
        lambda d: d * q2 / g.safe_nu,  # radial / nu
        lambda d: d * g.qx,  # jx
        lambda d: d * g.qy,  # jy
    )


def eta22(spectrum: np.ndarray, qx: np.ndarray, qy: np.ndarray, rank: int):
    """Prescribed-rank GL eta22 (``spatial.py:156-231``; MATLAB ``green_laplace_eta22.m:1-79``).

    Returns the dimensionless analytic field eta22/h (complex, physical space).
    """
    g = Geometry(qx, qy)
    support = support_of(spectrum)
    if np.any(qx[support] <= 0) or np.any(g.q[support] <= 0):
        raise ValueError("strict-forward nonzero analytic eta1 support is required")
    check_alias_safe(support, 2)
    out_support = minkowski_support(support, 2)
    qp = peak_q_of(spectrum, support, g.q)
    lam = np.sqrt((2.0 * np.sqrt(qp * np.tanh(qp))) ** 2 - 2.0 * qp * np.tanh(2.0 * qp))
    if not np.isfinite(lam) or lam <= 0:
        raise ValueError("invalid determinant-root Green--Laplace scale")
    nodes, weights = gauss_laguerre(rank)
    shift = 0.5 * (float(np.min(g.nu[support])) + float(np.max(g.sqrt_a[out_support])) / 2.0)
    banks = _eta22_banks(g)
    acc = np.zeros_like(spectrum)
    for x, w in zip(nodes, weights):
        tau = x / lam
        damped = spectrum * np.exp(-tau * (g.nu - shift))
        v, v_nu, v_nu2, hx, hy, rad, jx, jy = (np.fft.ifft2(bank(damped)) for bank in banks)
        sd = 2.0 * v * v_nu2 + v_nu**2 - hx**2 - hy**2
        sk = 2.0 * v * rad + 2.0 * (hx * jx + hy * jy)
        coef = w * np.exp(x) / lam / 4.0 * np.exp(-2.0 * shift * tau)
        sh = sinh_over_root(g.sqrt_a, tau)
        sd_hat = np.fft.fft2(sd)
        sk_hat = np.fft.fft2(sk)
        sd_hat[~out_support] = 0.0
        sk_hat[~out_support] = 0.0
        sd_hat = zero_below_roundoff_floor(sd_hat, out_support)
        sk_hat = zero_below_roundoff_floor(sk_hat, out_support)
        acc += coef * (-g.a * sh * sd_hat + np.cosh(g.sqrt_a * tau) * sk_hat)
    audit = {
        "implementation": "prescribed-rank-green-laplace-eta22",
        "quadrature_rank": rank,
        "peak_depth_wavenumber": qp,
        "scale": float(lam),
        "balance_shift": shift,
    }
    return np.fft.ifft2(acc), audit


def _radial_channels(support: np.ndarray, nu: np.ndarray, count: int = 2):
    """Radial nu-channels with per-channel shifts (``spatial.py:322-346``)."""
    active = nu[support]
    edges = np.linspace(float(np.min(active)), float(np.max(active)), count + 1)
    masks, shifts = [], []
    for c in range(count):
        upper = (nu < edges[c + 1]) if c < count - 1 else (nu <= edges[c + 1])
        mask = support & (nu >= edges[c]) & upper
        if np.any(mask):
            masks.append(mask)
            shifts.append(0.5 * (float(np.min(nu[mask])) + float(np.max(nu[mask]))))
    hats = [np.fft.fft2(m.astype(float)) for m in masks]
    pair = [[np.real(np.fft.ifft2(hats[i] * hats[j])) > 0.5 for j in range(len(masks))]
            for i in range(len(masks))]
    return masks, shifts, pair


def psi22(spectrum: np.ndarray, qx: np.ndarray, qy: np.ndarray, *,
          allow_below_model_parent_domain: bool = False):
    """Dual-branch GL2+2 psi22 with radial balance (``spatial.py:234-414``).

    Returns the dimensionless analytic field psi22/(h sqrt(g h)).
    """
    g = Geometry(qx, qy)
    support = support_of(spectrum)
    if not np.any(support) or np.any(qx[support] <= 0) or np.any(g.q[support] <= 0):
        raise ValueError("strict-forward nonzero analytic eta1 support is required")
    below = bool(np.any(g.q[support] < 0.3))
    if below and not allow_below_model_parent_domain:
        raise ValueError("psi22 requires parent kh >= 0.3")
    below_mass = float(np.sum(np.abs(spectrum[g.q < 0.3]) ** 2)
                       / max(np.sum(np.abs(spectrum) ** 2), TINY))
    check_alias_safe(support, 2)
    out_support = minkowski_support(support, 2)
    masks, shifts, pair_supports = _radial_channels(support, g.nu, 2)
    qp = peak_q_of(spectrum, support, g.q)
    peak_nu = np.sqrt(qp * np.tanh(qp))
    peak_out = np.sqrt(2.0 * qp * np.tanh(2.0 * qp))
    scales = (2.0 * peak_nu - peak_out, 2.0 * peak_nu + peak_out)
    r2 = np.sqrt(2.0)
    nodes = np.array([2.0 - r2, 2.0 + r2])
    weights = np.array([nodes[0] / (4.0 * (r2 - 1.0) ** 2), nodes[1] / (4.0 * (r2 + 1.0) ** 2)])
    banks = _eta22_banks(g)
    resolvent = np.zeros_like(spectrum)
    for branch, lam, ksign in (("slow", scales[0], -1.0), ("fast", scales[1], 1.0)):
        if lam <= 0 or not np.isfinite(lam):
            raise ValueError("invalid dual-branch Green--Laplace scale")
        for x, w in zip(nodes, weights):
            tau = x / lam
            coef = w * np.exp(x) / lam / 8.0
            fields = []
            for mask, shift in zip(masks, shifts):
                chan = spectrum * mask * np.exp(-tau * (g.nu - shift))
                fields.append([np.fft.ifft2(bank(chan)) for bank in banks])
            response = np.zeros_like(spectrum)
            for i, left in enumerate(fields):
                for j, right in enumerate(fields):
                    # bank order: v, v_nu, v_nu2, hx, hy, radial, jx, jy
                    sd = (2.0 * left[0] * right[2] + left[1] * right[1]
                          - left[3] * right[3] - left[4] * right[4])
                    sk = 2.0 * left[0] * right[5] + 2.0 * (left[3] * right[6] + left[4] * right[7])
                    sd_hat = np.fft.fft2(sd)
                    sk_hat = np.fft.fft2(sk)
                    ssum = shifts[i] + shifts[j]
                    if branch == "slow":
                        factor = np.exp((g.sqrt_a - ssum) * tau)
                    else:
                        factor = np.exp(-(g.sqrt_a + ssum) * tau)
                    part = factor * (sd_hat + ksign * sk_hat / g.safe_nu)
                    part[~pair_supports[i][j]] = 0.0
                    response += part
            resolvent += 1j * coef * response
    eta11 = np.fft.ifft2(spectrum)
    phi1z = -1j * np.fft.ifft2(spectrum * g.nu)
    total = resolvent + np.fft.fft2(0.5 * eta11 * phi1z)
    total[~out_support] = 0.0
    audit = {
        "implementation": "dual-branch-green-laplace-psi22",
        "lambda_minus": float(scales[0]),
        "lambda_plus": float(scales[1]),
        "radial_balance_channel_count": len(masks),
        "channel_shifts": list(shifts),
        "below_model_parent_domain": below,
        "below_model_spectral_mass": below_mass,
    }
    return np.fft.ifft2(total), audit


# ---------------------------------------------------------------------------
# order three (the eta33 + psi33 graph)
# ---------------------------------------------------------------------------

INNER_RANKS = (4, 6, 8, 10, 12)
OUTER_RANKS = (3, 4, 6, 8, 10)


def _np_ffts():
    return np.fft.ifft2, np.fft.fft2


def _first_state(damped: np.ndarray, g: Geometry, ffts=None) -> dict:
    """12-field first-order state (``_order3.py:175-193``, multipliers ``:151-172``)."""
    ifft2, _ = ffts or _np_ffts()
    q2 = g.q**2
    bank = {
        "eta": None,
        "etax": 1j * g.qx,
        "etay": 1j * g.qy,
        "phix": g.qx / g.safe_nu,
        "phiy": g.qy / g.safe_nu,
        "phiz": -1j * g.nu,
        "phixz": g.nu * g.qx,
        "phiyz": g.nu * g.qy,
        "phizz": -1j * q2 / g.safe_nu,
        "phizzz": -1j * q2 * g.nu,
        "phitz": -g.a,
        "phitzz": -q2,
    }
    st = {k: ifft2(damped if m is None else m * damped) for k, m in bank.items()}
    st["eta_t"] = st["phiz"]
    st["phiz_t"] = st["phitz"]
    st["phizz_t"] = st["phitzz"]
    return st


def _pair_state(damped, g: Geometry, out_support, nodes, weights, lam2, shift2,
                ffts_for=None) -> dict:
    """Inner GL loop and the 9 pair fields (``_order3.py:196-272``).

    ``ffts_for(i)`` (precision experiments only) gives the (ifft2, fft2) pair
    of inner node i, ``ffts_for(None)`` that of the 9 pair-field transforms."""
    ffts_for = ffts_for or (lambda i: _np_ffts())
    q2 = g.q**2
    bank = (None, g.nu, g.nu**2, g.nu**3, g.qx / g.safe_nu, g.qy / g.safe_nu,
            g.qx, g.qy, q2 / g.safe_nu, q2, g.nu * g.qx, g.nu * g.qy)
    e_hat = np.zeros_like(damped)
    et_hat = np.zeros_like(damped)
    p_hat = np.zeros_like(damped)
    pt_hat = np.zeros_like(damped)
    for i, (x, w) in enumerate(zip(nodes, weights)):
        ifft2, fft2 = ffts_for(i)
        tau = x / lam2
        d2 = damped * np.exp(-tau * (g.nu - shift2))
        v, v1, v2, v3, hx, hy, jx, jy, rad, qq, njx, njy = (
            ifft2(d2 if m is None else d2 * m) for m in bank
        )
        sources = (
            2.0 * v * v2 + v1**2 - hx**2 - hy**2,
            2.0 * v * rad + 2.0 * (hx * jx + hy * jy),
            2.0 * v * v3 + 4.0 * v1 * v2 - 2.0 * hx * jx - 2.0 * hy * jy,
            2.0 * (v1 * rad + v * qq) + 2.0 * (jx**2 + hx * njx + jy**2 + hy * njy),
        )
        hats = []
        for src in sources:
            h = fft2(src)
            h[~out_support] = 0.0
            hats.append(h)
        sd, sk, sdt, skt = (zero_below_roundoff_floor(h, out_support) for h in hats)
        sh = sinh_over_root(g.sqrt_a, tau)
        ch = np.cosh(g.sqrt_a * tau)
        coef = w * np.exp(x) / lam2 * np.exp(-2.0 * shift2 * tau) / 4.0
        e_hat += coef * (-g.a * sh * sd + ch * sk)
        et_hat -= 1j * coef * (-g.a * sh * sdt + ch * skt)
        p_hat += 1j * coef * (ch * sd - sh * sk)
        pt_hat += coef * (ch * sdt - sh * skt)
    for h in (e_hat, et_hat, p_hat, pt_hat):
        h[~out_support] = 0.0
    et_hat = zero_below_roundoff_floor(et_hat, out_support)
    dx = 1j * g.qx
    dy = 1j * g.qy
    ifft2, _ = ffts_for(None)
    pair = {
        "eta": ifft2(e_hat),
        "etax": ifft2(dx * e_hat),
        "etay": ifft2(dy * e_hat),
        "phix": ifft2(dx * p_hat),
        "phiy": ifft2(dy * p_hat),
        "phiz": ifft2(g.a * p_hat),
        "phizz": ifft2(q2 * p_hat),
        "phitz": ifft2(g.a * pt_hat),
        "eta_t": ifft2(et_hat),
    }
    pair["phiz_t"] = pair["phitz"]
    return pair


def _cubic_forcing(f: dict, p: dict):
    """Kinematic/dynamic cubic forcing and surface Taylor contact (``_order3.py:76-102, 275-287``)."""
    k_pair = (f["phix"] * p["etax"] + f["phiy"] * p["etay"] + p["phix"] * f["etax"]
              + p["phiy"] * f["etay"] - f["eta"] * p["phizz"] - p["eta"] * f["phizz"])
    k_direct = (f["eta"] * (f["phixz"] * f["etax"] + f["phiyz"] * f["etay"])
                - 0.5 * f["eta"] ** 2 * f["phizzz"])
    d_pair = (f["eta"] * p["phitz"] + p["eta"] * f["phitz"] + f["phix"] * p["phix"]
              + f["phiy"] * p["phiy"] + f["phiz"] * p["phiz"])
    d_direct = (0.5 * f["eta"] ** 2 * f["phitzz"]
                + f["eta"] * (f["phix"] * f["phixz"] + f["phiy"] * f["phiyz"]
                              + f["phiz"] * f["phizz"]))
    contact = (0.5 * f["eta"] * p["phiz"] + 0.5 * p["eta"] * f["phiz"]
               + 0.125 * f["eta"] ** 2 * f["phizz"])
    contact_t = (0.5 * (f["eta_t"] * p["phiz"] + f["eta"] * p["phiz_t"])
                 + 0.5 * (p["eta_t"] * f["phiz"] + p["eta"] * f["phiz_t"])
                 + 0.25 * f["eta"] * f["eta_t"] * f["phizz"]
                 + 0.125 * f["eta"] ** 2 * f["phizz_t"])
    return k_direct / 4.0 + k_pair / 2.0, d_direct / 4.0 + d_pair / 2.0, contact, contact_t


def order3(spectrum: np.ndarray, qx: np.ndarray, qy: np.ndarray, *,
           inner_rank: int = 4, outer_rank: int = 4, outer_subset=None, ffts_for=None):
    """Nested no-Stokes GL eta33 + psi33 (``_order3.py:18-148``; MATLAB ``gl_no_stokes_eta33.m``).

    Returns (eta33/h, psi33/(h sqrt(gh)), audit), complex physical fields.
    ``outer_subset`` (bench sampling only) restricts the outer GL loop to the
    listed node indices, i.e. evaluates that fraction of the graph.
    ``ffts_for(j, i)`` (precision experiments only) gives the (ifft2, fft2)
    pair used by outer node j's inner node i, and ``ffts_for(j, None)`` the
    one of outer node j's own transforms (first-order state, pair fields,
    forcing); the default is numpy's FP64 pair everywhere.
    """
    ffts_for = ffts_for or (lambda j, i: _np_ffts())
    if inner_rank not in INNER_RANKS or outer_rank not in OUTER_RANKS:
        raise ValueError("unsupported inner or outer third-order GL rank")
    g = Geometry(qx, qy)
    support = support_of(spectrum)
    if not np.any(support) or np.any(qx[support] <= 0) or np.any(g.q[support] <= 0.5):
        raise ValueError("third-order reconstruction requires strict-forward parent kh > 0.5")
    check_alias_safe(support, 3)
    hat = np.fft.fft2(support.astype(float))
    s2 = np.real(np.fft.ifft2(hat**2)) > 0.5
    s3 = np.real(np.fft.ifft2(hat**3)) > 0.5
    nu_min = float(np.min(g.nu[support]))
    shift2 = 0.5 * (nu_min + float(np.max(g.sqrt_a[s2])) / 2.0)
    shift3 = 0.5 * (nu_min + float(np.max(g.sqrt_a[s3])) / 3.0)
    qp = peak_q_of(spectrum, support, g.q)
    peak_nu = np.sqrt(qp * np.tanh(qp))
    lam2 = 2.0 * peak_nu - np.sqrt(2.0 * qp * np.tanh(2.0 * qp))
    lam3 = 3.0 * peak_nu - np.sqrt(3.0 * qp * np.tanh(3.0 * qp))
    if lam2 <= 0 or lam3 <= 0:
        raise ValueError("invalid third-order Green--Laplace scales")
    inodes, iweights = gauss_laguerre(inner_rank)
    onodes, oweights = gauss_laguerre(outer_rank)
    eta_hat = np.zeros_like(spectrum)
    psi_hat = np.zeros_like(spectrum)
    for j, (x, w) in enumerate(zip(onodes, oweights)):
        if outer_subset is not None and j not in outer_subset:
            continue
        tau = x / lam3
        damped = spectrum * np.exp(-tau * (g.nu - shift3))
        first = _first_state(damped, g, ffts_for(j, None))
        pair = _pair_state(damped, g, s2, inodes, iweights, lam2, shift2,
                           lambda i, j=j: ffts_for(j, i))
        fk, fd, c, ct = _cubic_forcing(first, pair)
        _, fft2 = ffts_for(j, None)
        hats = []
        for src in (fk, fd, c, ct):
            h = fft2(src)
            h[~s3] = 0.0
            hats.append(zero_below_roundoff_floor(h, s3))
        fk_hat, fd_hat, c_hat, ct_hat = hats
        fk_psi = zero_below_roundoff_floor(fk_hat + g.a * c_hat, s3)
        fd_psi = zero_below_roundoff_floor(fd_hat - ct_hat, s3)
        sh = sinh_over_root(g.sqrt_a, tau)
        ch = np.cosh(g.sqrt_a * tau)
        coef = w * np.exp(x) / lam3 * np.exp(-3.0 * shift3 * tau)
        eta_hat += coef * (g.a * sh * fd_hat - 1j * ch * fk_hat)
        psi_hat += coef * (-1j * ch * fd_psi - sh * fk_psi)
    eta_hat[~s3] = 0.0
    psi_hat[~s3] = 0.0
    audit = {
        "implementation": "nested-no-stokes-green-laplace-order3",
        "inner_quadrature_rank": inner_rank,
        "outer_quadrature_rank": outer_rank,
        "inner_scale": float(lam2),
        "outer_scale": float(lam3),
        "inner_balance_shift": shift2,
        "outer_balance_shift": shift3,
        "peak_depth_wavenumber": qp,
    }
    return np.fft.ifft2(eta_hat), np.fft.ifft2(psi_hat), audit


# ---------------------------------------------------------------------------
# first order, input deposit and the two public calling patterns
# ---------------------------------------------------------------------------


def first_order(spectrum: np.ndarray, qx, qy):
    """eta11/h and psi11/(h sqrt(gh)) (``spatial.py:74-79``; ``gl_spectral_surface.m:26-31``)."""
    g = Geometry(qx, qy)
    eta11 = np.fft.ifft2(spectrum)
    psi_hat = np.zeros_like(spectrum)
    nz = g.nu > 0
    psi_hat[nz] = -1j * spectrum[nz] / g.nu[nz]
    return eta11, np.fft.ifft2(psi_hat)


def matlab_round(values: np.ndarray) -> np.ndarray:
    """MATLAB ``round``: half away from zero."""
    return np.sign(values) * np.floor(np.abs(values) + 0.5)


def deposit_modes(a, b, kx, ky, omega, h, lx, ly, nx, ny, t, grid_tolerance=1.0e-10):
    """Deposit ``N^2 (a + i b)/h e^{-i omega t}`` on the FFT grid.

    Restates ``deposit_analytic_input`` (``src/gl_spectral_surface.m:123-149``):
    off-grid and Nyquist modes raise, coincident modes add.
    """
    dkx = 2.0 * np.pi / lx
    dky = 2.0 * np.pi / ly
    spectrum = np.zeros((ny, nx), dtype=complex)
    scale = float(nx * ny)
    for ai, bi, kxi, kyi, wi in zip(a, b, kx, ky, omega):
        mx = int(matlab_round(np.array(kxi / dkx)))
        my = int(matlab_round(np.array(kyi / dky)))
        tol = grid_tolerance * max(1.0, float(np.hypot(kxi, kyi)))
        if abs(kxi - mx * dkx) > tol or abs(kyi - my * dky) > tol:
            raise ValueError("Every component must lie on the requested FFT grid.")
        if abs(mx) >= nx / 2 or abs(my) >= ny / 2:
            raise ValueError("An input component reaches or exceeds a Nyquist boundary.")
        amp = complex(ai / h, bi / h)
        spectrum[my % ny, mx % nx] += scale * amp * np.exp(-1j * wi * t)
    return spectrum


def spectral_coefficients(order, g, h, a, b, kx, ky, ux=0.0, uy=0.0, options=None):
    """Validation and omega/peak bookkeeping (``src/gl_spectral_coefficients.m:1-88``)."""
    opts = {"sector": "pure-sum", "eta22_rank": 6, "peak_wavenumber": None,
            "allow_below_model_parent_domain": False, "grid_tolerance": 1e-10}
    for key, value in (options or {}).items():
        if key not in opts:
            raise ValueError(f"Unknown Green--Laplace option: {key}")
        opts[key] = value
    if order not in (1, 2, 3):
        raise ValueError("order must be 1, 2, or 3")
    if ux != 0 or uy != 0:
        raise ValueError("only Ux=Uy=0 is certified")
    a, b, kx, ky = (np.asarray(v, dtype=float).ravel() for v in (a, b, kx, ky))
    if a.size == 0 or not (a.size == b.size == kx.size == ky.size):
        raise ValueError("a, b, kx, and ky must be nonempty vectors of equal length.")
    if not np.all(np.isfinite(np.concatenate([a, b, kx, ky]))) or np.any(np.hypot(kx, ky) <= 0):
        raise ValueError("Component amplitudes and nonzero wavenumbers must be finite.")
    if np.any(kx <= 0):
        raise ValueError("The released GL graphs require strict-forward support kx>0.")
    amp = np.hypot(a, b)
    if not np.any(amp > 0):
        raise ValueError("At least one input amplitude is required.")
    k = np.hypot(kx, ky)
    pq = h * k
    if order >= 2 and np.any(pq < 0.3) and not opts["allow_below_model_parent_domain"]:
        raise ValueError("Order-two surface-potential reconstruction requires kh>=0.3.")
    if order >= 3 and np.any(pq <= 0.5):
        raise ValueError("Order-three reconstruction requires every parent kh>0.5.")
    omega = np.sqrt(g * k * np.tanh(h * k))
    if opts["peak_wavenumber"] is None:
        peak_k = float(k[int(np.argmax(amp**2))])
    else:
        peak_k = float(opts["peak_wavenumber"])
    return {"order": int(order), "g": float(g), "h": float(h), "a": a, "b": b, "kx": kx, "ky": ky,
            "omega": omega, "peak_wavenumber": peak_k, "peak_depth": h * peak_k, "options": opts}


def spectral_surface(coeffs: dict, lx, ly, nx, ny, t):
    """Two-stage surface evaluation (``src/gl_spectral_surface.m:1-103``) on the Python internals.

    Returns a dict of physical component fields (complex ``*_plus`` and real parts).
    """
    h, grav = coeffs["h"], coeffs["g"]
    kxg, kyg = fft_wavenumber_grid(lx, ly, nx, ny)
    s = deposit_modes(coeffs["a"], coeffs["b"], coeffs["kx"], coeffs["ky"], coeffs["omega"], h,
                      lx, ly, nx, ny, t, coeffs["options"]["grid_tolerance"])
    return evaluate_spectrum(s, h * kxg, h * kyg, depth=h, gravity=grav, order=coeffs["order"],
                             eta22_rank=coeffs["options"]["eta22_rank"],
                             allow_below=coeffs["options"]["allow_below_model_parent_domain"])


def evaluate_spectrum(s, qx, qy, *, depth, gravity, order, eta22_rank=6, allow_below=False):
    """All components from a deposited analytic spectrum (``spatial.py:74-124``)."""
    pscale = depth * np.sqrt(gravity * depth)
    e11, p11 = first_order(s, qx, qy)
    comp: dict[str, Any] = {"eta11_plus": depth * e11, "psi11_plus": pscale * p11}
    audits: dict[str, Any] = {}
    if order >= 2:
        e22, a22 = eta22(s, qx, qy, eta22_rank)
        p22, b22 = psi22(s, qx, qy, allow_below_model_parent_domain=allow_below)
        comp["eta22_plus"] = depth * e22
        comp["psi22_plus"] = pscale * p22
        audits["eta22"], audits["psi22"] = a22, b22
    if order >= 3:
        e33, p33, a33 = order3(s, qx, qy)
        comp["eta33_plus"] = depth * e33
        comp["psi33_plus"] = pscale * p33
        audits["order3"] = a33
    for key in list(comp):
        comp[key[:-5]] = np.real(comp[key])
    comp["_audits"] = audits
    return comp


def analytic_spectrum(eta1: np.ndarray, depth: float, kx: np.ndarray, tolerance: float = 1e-11):
    """Strict-forward analytic spectrum of a real snapshot (``_spectral.py:19-49``)."""
    if eta1.ndim != 2 or eta1.shape != kx.shape or not np.all(np.isfinite(eta1)):
        raise ValueError("eta1 must be a finite two-dimensional grid")
    raw = np.fft.fft2(eta1 / depth)
    scale = max(float(np.max(np.abs(raw))), TINY)
    zero_line = np.abs(kx) <= 32.0 * EPS * max(1.0, np.max(np.abs(kx)))
    if np.max(np.abs(raw[zero_line]), initial=0.0) > tolerance * scale:
        raise ValueError("eta1 contains a non-negligible kx=0 component")
    s = np.zeros_like(raw, dtype=np.complex128)
    s[kx > 0] = 2.0 * raw[kx > 0]
    rec = np.real(depth * np.fft.ifft2(s))
    err = float(np.linalg.norm(rec - eta1) / max(np.linalg.norm(eta1), TINY))
    if err > tolerance:
        raise ValueError("eta1 is not consistent with the declared strict-forward x propagation")
    return s, err


def reconstruct_directional_field(eta1, *, lx, ly, depth, gravity=9.81, time=0.0, order=2,
                                  eta22_rank=6, allow_below_model_parent_domain=False):
    """Real-grid entry (``spatial.py:33-153``): returns the component dict."""
    field_ = np.asarray(eta1, dtype=float)
    ny, nx = field_.shape
    kx, ky = fft_wavenumber_grid(lx, ly, nx, ny)
    s0, _ = analytic_spectrum(field_, depth, kx)
    qx, qy = depth * kx, depth * ky
    q = np.hypot(qx, qy)
    nu = np.sqrt(q * np.tanh(q))
    s = s0 * np.exp(-1j * np.sqrt(gravity / depth) * nu * time)
    return evaluate_spectrum(s, qx, qy, depth=depth, gravity=gravity, order=order,
                             eta22_rank=eta22_rank, allow_below=allow_below_model_parent_domain)
