"""Seeded synthetic directional sea states on the FFT lattice.

The reference publishes no sea-state generator for its spatial API (its MATLAB
generator, ``paper/internal/generate_directional_input.m``, is dimensionless
with Gaussian spreading).  The workloads here are drawn from a JONSWAP
frequency spectrum with ``cos^(2s)(theta/2)`` spreading about +x:

* candidate cells: ``mx >= 1`` (strict-forward), ``|m| < N/(2*order)``
  (alias-safe for the requested order) and parent ``kh`` inside the order's
  model domain (``kh >= 0.3`` for order 2, ``kh > 0.5`` for order 3);
* JONSWAP ``S(omega)`` (gamma, sigma 0.07/0.09) converted to a wavenumber
  density with the finite-depth group velocity, times the spreading;
* the M densest cells are kept and the variance normalised to ``Hs^2/16``;
* ``a, b = default_rng(seed).standard_normal(M) * sqrt(S dkx dky)``.

Frequencies come from the finite-depth dispersion relation in FP64.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class SeaState:
    """First-order components on the 2*pi/L lattice (physical units)."""

    a: np.ndarray
    b: np.ndarray
    kx: np.ndarray
    ky: np.ndarray
    depth: float
    gravity: float
    lx: float
    ly: float
    nx: int
    ny: int

    @property
    def modes(self) -> int:
        return int(self.a.size)


def jonswap_sea_state(*, n: int, length: float, depth: float, hs: float, tp: float, modes: int,
                      seed: int, order: int = 3, gravity: float = 9.81, gamma: float = 3.3,
                      spreading: float = 10.0) -> SeaState:
    """Build a seeded JONSWAP + cos^(2s) sea state for an ``n x n`` grid of side ``length``."""
    if n % 2 or n < 8:
        raise ValueError("grid size must be even and >= 8")
    dk = 2.0 * np.pi / length
    lim = n / (2.0 * order)
    m = np.arange(-(n // 2) + 1, n // 2)
    mx, my = np.meshgrid(m, m)
    kx = mx * dk
    ky = my * dk
    k = np.hypot(kx, ky)
    kh_floor = 0.3 if order <= 2 else 0.5
    ok = (mx >= 1) & (np.abs(mx) < lim) & (np.abs(my) < lim)
    ok &= (k * depth > kh_floor) if order >= 3 else (k * depth >= kh_floor)
    ks = np.where(ok, k, 1.0)
    omega = np.sqrt(gravity * ks * np.tanh(ks * depth))
    wp = 2.0 * np.pi / tp
    sigma = np.where(omega <= wp, 0.07, 0.09)
    s_omega = (gravity**2 / omega**5 * np.exp(-1.25 * (wp / omega) ** 4)
               * gamma ** np.exp(-((omega - wp) ** 2) / (2.0 * sigma**2 * wp**2)))
    kd = np.minimum(2.0 * ks * depth, 700.0)
    cg = 0.5 * omega / ks * (1.0 + kd / np.sinh(kd))
    theta = np.arctan2(ky, kx)
    density = np.where(ok, s_omega * cg / ks * np.cos(theta / 2.0) ** (2.0 * spreading), 0.0)
    order_idx = np.argsort(density.ravel(), kind="stable")[::-1][:modes]
    if order_idx.size < modes or density.ravel()[order_idx[-1]] <= 0:
        raise ValueError("not enough admissible lattice cells for the requested mode count")
    s = density.ravel()[order_idx]
    s = s * (hs**2 / 16.0) / (np.sum(s) * dk * dk)
    rng = np.random.default_rng(seed)
    amp = np.sqrt(s * dk * dk)
    a = rng.standard_normal(modes) * amp
    b = rng.standard_normal(modes) * amp
    return SeaState(a=a, b=b, kx=kx.ravel()[order_idx].astype(float),
                    ky=ky.ravel()[order_idx].astype(float), depth=float(depth),
                    gravity=float(gravity), lx=float(length), ly=float(length), nx=n, ny=n)


def config1(seed: int = 0) -> SeaState:
    """Order-2 workload: h=20 m, L=512 m, 256^2, 400 modes, Hs=2 m, Tp=10 s."""
    return jonswap_sea_state(n=256, length=512.0, depth=20.0, hs=2.0, tp=10.0, modes=400,
                             seed=seed, order=2)


def config2(seed: int = 0) -> SeaState:
    """Order-3 workload: h=30 m, L=1024 m, 1024^2, 4096 modes, Hs=3 m, Tp=10 s."""
    return jonswap_sea_state(n=1024, length=1024.0, depth=30.0, hs=3.0, tp=10.0, modes=4096,
                             seed=seed, order=3)


def config4(seed: int = 0) -> SeaState:
    """Adjoint-fit workload: h=25 m, L=512 m, 512^2, 2048 modes, Hs=2.5 m, Tp=10 s."""
    return jonswap_sea_state(n=512, length=512.0, depth=25.0, hs=2.5, tp=10.0, modes=2048,
                             seed=seed, order=3)


def small_order3(seed: int = 0, n: int = 64, modes: int = 24, depth: float = 30.0,
                 length: float | None = None) -> SeaState:
    """A small order-3 sea state for parity tests (defaults: 64^2, 24 modes)."""
    length = float(length if length is not None else 2.0 * n)
    return jonswap_sea_state(n=n, length=length, depth=depth, hs=2.0, tp=8.0, modes=modes,
                             seed=seed, order=3)


def config5_case(*, peak_kh: float = 1.5, steepness: float = 0.08, modes: int = 1024,
                 n: int = 1024, seed: int = 0, sigma: float = 0.35, spreading: float = 10.0):
    """Dimensionless order-4 sea state (g = h = 1) on an n x n grid.

    The lattice step is chosen so the peak sits at |m| = 50 (dk = peak_kh / 50),
    cells with kh in [0.8, 3] and 4 |m| < n / 2 (the quartic alias guard) are
    admissible, their density is a Gaussian in kh about ``peak_kh`` (width
    ``sigma``) times cos^(2 s)(theta / 2) about +x, and the ``modes`` densest
    cells are kept (deterministic top-density cells, like the reference's
    dimensionless generator).  Amplitudes |c| ~ sqrt(density), phases uniform
    from ``seed``, scaled so that steepness = k_p sqrt(sum |c|^2) (k_p |c| for
    one mode).  Returns a wit.WitInput with one amplitude case."""
    from .wit import WitInput

    dk = peak_kh / 50.0
    lim = n // 8
    m = np.arange(-lim + 1, lim)
    mx, my = np.meshgrid(m, m)
    k = dk * np.hypot(mx, my)
    theta = np.arctan2(my, mx)
    ok = (mx >= 1) & (k >= 0.8) & (k <= 3.0)
    dens = np.where(ok, np.exp(-0.5 * ((k - peak_kh) / sigma) ** 2)
                    * np.cos(theta / 2.0) ** (2.0 * spreading), 0.0)
    idx = np.argsort(dens.ravel(), kind="stable")[::-1][:modes]
    if idx.size < modes or dens.ravel()[idx[-1]] <= 0:
        raise ValueError("not enough admissible lattice cells for the requested mode count")
    rng = np.random.default_rng(seed)
    amp = np.sqrt(dens.ravel()[idx]) * np.exp(2j * np.pi * rng.random(modes))
    amp *= steepness / (peak_kh * np.sqrt(np.sum(np.abs(amp) ** 2)))
    cells = np.stack([mx.ravel()[idx], my.ravel()[idx]], axis=1).astype(np.int32)
    return WitInput(modes=cells, amplitudes=amp[None, :], nx=n, ny=n, gravity=1.0, depth=1.0,
                    dkx=dk, dky=dk, threshold=1e-6)


def largest_modes(inp, count: int):
    """The ``count`` modes of largest amplitude (their original order kept)."""
    from .wit import WitInput

    keep = np.sort(np.argsort(-np.abs(inp.amplitudes[0]), kind="stable")[:count])
    return WitInput(modes=inp.modes[keep], amplitudes=inp.amplitudes[:, keep], nx=inp.nx,
                    ny=inp.ny, gravity=inp.gravity, depth=inp.depth, dkx=inp.dkx, dky=inp.dky,
                    threshold=inp.threshold)
