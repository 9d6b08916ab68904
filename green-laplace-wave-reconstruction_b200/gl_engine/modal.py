"""Single-direction time reconstruction on a one-dimensional modal grid.

Mirror of the reference's time-series interface
(``python/src/green_laplace/modal_time.py:26-214``,
``reconstruct_unidirectional_modal_timeseries``; ``temporal.py:19-60``,
``reconstruct_unidirectional_timeseries``), evaluated by the engine's CUDA
kernels through ``gl_modal_level`` / ``gl_eta20_level`` /
``gl_series_synthesize``.  The host side does what the reference's driver
does around its graph: checks the record, takes its DFT band, solves the
dispersion relation, spreads the amplitudes onto the modal axis (index and
weight bookkeeping) and walks the modal-points ladder until two levels agree.
"""

from __future__ import annotations

import ctypes as C
from collections.abc import Sequence
from dataclasses import dataclass
from time import perf_counter
from typing import Any

import numpy as np
import torch

from . import _lib, api

TINY = float(np.finfo(float).tiny)


@dataclass(frozen=True)
class ModalTimeSeriesResult:
    time: np.ndarray
    eta: np.ndarray
    components: dict
    audit: dict


TimeSeriesResult = ModalTimeSeriesResult


def _ladder(modal_points) -> tuple[int, ...]:
    ladder = (modal_points,) if isinstance(modal_points, (int, np.integer)) else tuple(
        int(v) for v in modal_points)
    if (not ladder or any(v < 16 or v % 2 for v in ladder)
            or any(b <= a for a, b in zip(ladder, ladder[1:]))):
        raise ValueError("modal_points must be an increasing sequence of even integers")
    return ladder


def _deposit(amps, work_bins, q, axis, step, width, shift_rows):
    """Two-neighbour linear spread (``modal_time.py:375-386``), duplicates summed
    in the reference's order; rows moved to numpy's ifftshift order."""
    pos = (q - axis[0]) / step
    lo = np.clip(np.floor(pos).astype(int), 0, axis.size - 2)
    hi = lo + 1
    w_hi = np.clip(pos - lo, 0.0, 1.0)
    w_lo = 1.0 - w_hi
    acc: dict[int, complex] = {}
    for rows, wts in ((lo, w_lo), (hi, w_hi)):
        for r, b, v in zip(rows, work_bins, amps * wts):
            k = int(shift_rows(r)) * width + int(b)
            acc[k] = acc.get(k, 0j) + v
    mass = np.abs(amps) ** 2
    err = np.concatenate((np.abs(axis[lo] - q) / q, np.abs(axis[hi] - q) / q))
    wts = np.concatenate((mass * w_lo, mass * w_hi))
    rms = float(np.sqrt(np.sum(wts * err**2) / max(np.sum(wts), TINY)))
    idx = np.fromiter(acc.keys(), dtype=np.int64, count=len(acc))
    val = np.array(list(acc.values()), dtype=np.complex128)
    return idx, val, rms


class _Device:
    def __init__(self, device):
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise api.GLError("green_laplace:Device", "the GL engine runs on CUDA devices only")
        self.lib = _lib.load()

    def t(self, a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device, dtype)

    @property
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def synth(self, count, bins, coef, real_only):
        bins = np.asarray(bins, dtype=np.int32)
        dc = self.t(np.ascontiguousarray(np.asarray(coef, dtype=np.complex128)).view(np.float64),
                    torch.float64)
        db = self.t(bins, torch.int32)
        out = torch.empty(count if real_only else 2 * count, dtype=torch.float64, device=self.device)
        api._engine_call(self.lib.gl_series_synthesize(
            count, int(bins.size), C.c_void_p(db.data_ptr()), C.c_void_p(dc.data_ptr()),
            C.c_void_p(out.data_ptr()), int(bool(real_only)), C.c_void_p(self.stream)))
        res = out.cpu().numpy()
        return res if real_only else res.view(np.complex128)


def _rule(rank):
    nodes, weights = api.gauss_laguerre_rule(rank)
    return np.ascontiguousarray(nodes, dtype=float), np.ascontiguousarray(weights, dtype=float)


def _modal_level(dev: _Device, amps, bins, q, *, count, dt, depth, gravity, peak_q, rank, order,
                 points, limit):
    b0 = int(np.min(bins))
    wb = bins - b0
    wmax = int(np.max(wb))
    width = order * wmax + 1
    if width > count:
        raise ValueError("the nonlinear output band does not fit in the time record")
    if limit is None:
        limit = (order + 0.05) * float(np.max(np.abs(q))) / (1 - 2 / points)
    else:
        limit = float(limit)
        if limit <= order * float(np.max(np.abs(q))):
            raise ValueError("modal_limit must exceed the requested nonlinear output support")
    step = 2 * limit / points
    axis = np.arange(-points / 2, points / 2) * step
    idx, val, rms = _deposit(amps, wb, q, axis, step, width, lambda r: (r + points // 2) % points)
    nodes, weights = _rule(rank)
    pnu = np.sqrt(peak_q * np.tanh(peak_q))
    desc = _lib.ModalDesc(
        points=points, width=width, order=order, base_bin=b0, count=count, q_step=step,
        freq_step=2 * np.pi / (count * dt) * np.sqrt(depth / gravity), depth=depth,
        scale22=float(np.sqrt(4 * peak_q * np.tanh(peak_q) - 2 * peak_q * np.tanh(2 * peak_q))),
        lambda2=float(2 * pnu - np.sqrt(2 * peak_q * np.tanh(2 * peak_q))),
        lambda3=float(3 * pnu - np.sqrt(3 * peak_q * np.tanh(3 * peak_q))), rank=rank,
        nodes=nodes.ctypes.data_as(C.POINTER(C.c_double)),
        weights=weights.ctypes.data_as(C.POINTER(C.c_double)))
    size = C.c_size_t()
    api._engine_call(dev.lib.gl_modal_workspace_size(C.byref(desc), C.byref(size)))
    with torch.cuda.device(dev.device):
        ws = torch.empty(int(size.value) + 256, dtype=torch.uint8, device=dev.device)
        wsp = (ws.data_ptr() + 255) & ~255
        d_idx = dev.t(idx, torch.int64)
        d_val = dev.t(val.view(np.float64), torch.float64)
        e22 = torch.empty(2 * count, dtype=torch.float64, device=dev.device)
        e33 = torch.empty(2 * count, dtype=torch.float64, device=dev.device) if order >= 3 else None
        api._engine_call(dev.lib.gl_modal_level(
            C.byref(desc), int(idx.size), C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_val.data_ptr()),
            C.c_void_p(e22.data_ptr()), C.c_void_p(e33.data_ptr() if e33 is not None else 0),
            C.c_void_p(wsp), C.c_size_t(int(size.value)), C.c_void_p(dev.stream)))
        out22 = e22.cpu().numpy().view(np.complex128)
        out33 = e33.cpu().numpy().view(np.complex128) if e33 is not None else None
    return out22, out33, {"modal_points": points, "modal_limit": float(abs(axis[0])),
                          "quadrature_rank": rank, "base_bin": b0, "work_frequency_count": width,
                          "wavevector_projection_rms_relative": rms}


def _hermitian_project(c):
    out = c.copy()
    n = out.size
    for k in range(1, (n - 1) // 2 + 1):
        m = (out[k] + np.conj(out[-k])) / 2.0
        out[k] = m
        out[-k] = np.conj(m)
    out[0] = np.real(out[0])
    if n % 2 == 0:
        out[n // 2] = np.real(out[n // 2])
    return out


def unidirectional_eta20(dev: _Device, amps, omega, q, times, *, depth, gravity, rank=16, nx=128,
                         ny=16):
    """Difference-frequency eta20 (``_eta20.py:13-151``) on the GPU."""
    if rank not in (6, 12, 16):
        raise ValueError("eta20 rank must be 6, 12, or 16")
    if nx < 16 or ny < 16 or nx % 2 or ny % 2:
        raise ValueError("eta20 modal-grid sizes must be even and at least 16")
    count = times.size
    dt = float(np.mean(np.diff(times)))
    bins = np.rint(omega * count * dt / (2.0 * np.pi)).astype(int)
    if np.any(bins < 1) or not np.allclose(omega, 2.0 * np.pi * bins / (count * dt), rtol=1e-10,
                                           atol=1e-12):
        raise ValueError("eta20 input frequencies must lie on temporal DFT bins")
    b0 = int(np.min(bins))
    wb = bins - b0
    span = int(np.max(wb))
    width = 2 * span + 1
    energy = np.abs(amps) ** 2
    esum = float(np.sum(energy))
    mean_q = float(np.sum(q * energy) / esum)
    dq = float(np.sqrt(2.0 * np.sum((q - mean_q) ** 2 * energy) / esum))
    audit = {"implementation": "modal-grid-green-laplace-eta20", "quadrature_rank": rank,
             "interaction_enumeration": False}
    if dq <= 64.0 * np.finfo(float).eps * max(1.0, float(np.max(q))):
        audit["status"] = "degenerate-zero-difference-output"
        return np.zeros(count), audit
    lim_x = (2 + 0.05) * float(np.max(np.abs(q))) / (1.0 - 2.0 / nx)
    sx = 2.0 * lim_x / nx
    ax_x = np.arange(-nx / 2, nx / 2) * sx
    lim_y = (2.05 * float(np.max(q))) / (1.0 - 2.0 / ny)
    sy = 2.0 * lim_y / ny
    ax_y = np.arange(-ny / 2, ny / 2) * sy

    def bracket(value, axis, step):
        pos = (value - axis[0]) / step
        lo = np.clip(np.floor(pos).astype(int), 0, axis.size - 2)
        w_hi = np.clip(pos - lo, 0.0, 1.0)
        return lo, lo + 1, 1.0 - w_hi, w_hi

    ix0, ix1, wx0, wx1 = bracket(q, ax_x, sx)
    iy0, iy1, wy0, wy1 = bracket(np.zeros_like(q), ax_y, sy)
    acc: dict[int, complex] = {}
    for ix, wx in ((ix0, wx0), (ix1, wx1)):
        for iy, wy in ((iy0, wy0), (iy1, wy1)):
            for a, b, c, v in zip(iy, ix, wb, amps * wx * wy):
                r = ((int(a) + ny // 2) % ny) * nx + (int(b) + nx // 2) % nx
                k = r * width + int(c)
                acc[k] = acc.get(k, 0j) + v
    idx = np.fromiter(acc.keys(), dtype=np.int64, count=len(acc))
    val = np.array(list(acc.values()), dtype=np.complex128)
    nodes, weights = _rule(rank)
    desc = _lib.Eta20Desc(nx=nx, ny=ny, span=span, base_bin=b0, count=count, qx_step=sx, qy_step=sy,
                          freq_step=2.0 * np.pi / (count * dt) * np.sqrt(depth / gravity), depth=depth,
                          dq=dq, rank=rank, nodes=nodes.ctypes.data_as(C.POINTER(C.c_double)),
                          weights=weights.ctypes.data_as(C.POINTER(C.c_double)))
    size = C.c_size_t()
    api._engine_call(dev.lib.gl_eta20_workspace_size(C.byref(desc), C.byref(size)))
    with torch.cuda.device(dev.device):
        ws = torch.empty(int(size.value) + 256, dtype=torch.uint8, device=dev.device)
        wsp = (ws.data_ptr() + 255) & ~255
        d_idx = dev.t(idx, torch.int64)
        d_val = dev.t(val.view(np.float64), torch.float64)
        coef = torch.empty(2 * width, dtype=torch.float64, device=dev.device)
        api._engine_call(dev.lib.gl_eta20_level(
            C.byref(desc), int(idx.size), C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_val.data_ptr()),
            C.c_void_p(coef.data_ptr()), C.c_void_p(wsp), C.c_size_t(int(size.value)),
            C.c_void_p(dev.stream)))
        raw = coef.cpu().numpy().view(np.complex128)
    signed = np.concatenate((np.arange(0, span + 1), np.arange(-span, 0)))
    coefficients = np.zeros(count, dtype=np.complex128)
    for k, sb in enumerate(signed):
        coefficients[sb % count] = raw[k]
    coefficients = _hermitian_project(coefficients)
    nz = np.flatnonzero(coefficients)
    eta20 = dev.synth(count, nz, coefficients[nz], True)
    audit.update({"modal_grid": [ny, nx], "delta_q_rms_pair": dq,
                  "strict_zero_spatial_mode": "excluded"})
    return eta20, audit


def reconstruct_unidirectional_modal_timeseries(
        eta1, time, *, depth: float, gravity: float = 9.81, omega_max: float | None = None,
        energy_fraction: float = 0.999, quadrature_rank: int = 8, order: int = 3,
        modal_points: int | Sequence[int] = (2048, 4096, 8192, 16384, 32768, 65536),
        modal_limit: float | None = None, relative_tolerance: float = 1.0e-3,
        include_eta20: bool = True, eta20_rank: int = 16, eta20_grid: tuple[int, int] = (128, 16),
        device=None) -> ModalTimeSeriesResult:
    """Reconstruct a single-direction record with the direct modal resolvent
    (``modal_time.py:26-214``) on the GPU."""
    started = perf_counter()
    values = np.asarray(eta1, dtype=float).reshape(-1)
    times = np.asarray(time, dtype=float).reshape(-1)
    if values.size != times.size or values.size < 9:
        raise ValueError("eta1 and time must have the same length of at least nine")
    if depth <= 0 or gravity <= 0 or order not in (2, 3):
        raise ValueError("depth and gravity must be positive and order must be 2 or 3")
    ladder = _ladder(modal_points)
    if relative_tolerance <= 0:
        raise ValueError("relative_tolerance must be positive")
    if order == 3 and quadrature_rank not in (4, 6, 8, 10):
        raise ValueError("third-order modal reconstruction supports rank 4, 6, 8, or 10")
    count = values.size
    dt = float(np.mean(np.diff(times)))
    expected = times[0] + np.arange(count) * dt
    deviation = float(np.max(np.abs(times - expected)))
    if dt <= 0 or deviation > max(1e-10, 1024 * np.finfo(float).eps * max(1.0, times[-1] - times[0])):
        raise ValueError("a uniformly increasing time record is required")
    period = count * dt
    pos = (count - 1) // 2
    cand = np.arange(1, pos + 1)
    dft = np.fft.fft(values) / count
    energy = np.abs(dft[cand]) ** 2
    total = float(np.sum(energy))
    if total == 0:
        raise ValueError("eta1 has no positive-frequency content")
    cum = np.cumsum(energy) / total
    top = int(cand[min(int(np.searchsorted(cum, energy_fraction)), cand.size - 1)])
    top = min(top, pos // order)
    if omega_max is not None:
        top = min(top, int(np.floor(omega_max * period / (2 * np.pi))))
    if top < 1:
        raise ValueError("the selected eta1 frequency band is empty")
    bins = np.arange(1, top + 1)
    omega = 2 * np.pi * bins / period
    amps = 2 * np.conj(dft[bins])
    dev = _Device(device)
    eta11 = dev.synth(count, bins, amps, True)
    q = np.asarray(api.dimensionless_wavenumber_from_frequency(omega, depth=depth, gravity=gravity),
                   dtype=float)
    peak_q = float(q[int(np.argmax(np.abs(amps)))])

    prev = None
    levels = []
    converged = False
    e22 = e33 = None
    modal_audit = None
    for pts in ladder:
        t0 = perf_counter()
        e22, e33, modal_audit = _modal_level(dev, amps, bins, q, count=count, dt=dt, depth=depth,
                                             gravity=gravity, peak_q=peak_q, rank=quadrature_rank,
                                             order=order, points=pts, limit=modal_limit)
        cur = (e22,) if e33 is None else (e22, e33)
        changes = None
        if prev is not None:
            changes = tuple(float(np.linalg.norm(a - b) / np.linalg.norm(a)) for a, b in zip(cur, prev))
            converged = max(changes) <= relative_tolerance
        levels.append({"modal_points": pts, "seconds": perf_counter() - t0,
                       "eta22_change": None if changes is None else changes[0],
                       "eta33_change": None if changes is None or e33 is None else changes[1],
                       "wavevector_projection_rms_relative":
                           modal_audit["wavevector_projection_rms_relative"]})
        prev = cur
        if converged:
            break
    comps: dict[str, Any] = {"eta11": eta11, "eta22": np.real(e22), "eta22_analytic": e22}
    eta_total = eta11 + np.real(e22)
    if e33 is not None:
        comps["eta33"] = np.real(e33)
        comps["eta33_analytic"] = e33
        eta_total = eta_total + np.real(e33)
    if include_eta20:
        e20, a20 = unidirectional_eta20(dev, amps, omega, q, times, depth=depth, gravity=gravity,
                                        rank=eta20_rank, nx=eta20_grid[0], ny=eta20_grid[1])
        comps["eta20"] = e20
        eta_total = eta_total + e20
        modal_audit["eta20"] = a20
    modal_audit.update({
        "implementation": "one-dimensional-modal-green-laplace-time",
        "retained_positive_frequency_energy": float(np.sum(energy[:top]) / total),
        "input_projection_relative": float(np.linalg.norm(eta11 - values)
                                           / max(np.linalg.norm(values), TINY)),
        "solve_seconds": perf_counter() - started, "levels": levels, "converged": converged,
        "relative_tolerance": relative_tolerance, "auxiliary_space_domain": False,
        "interaction_enumeration": False, "stokes_correction": False,
        "engine": "gl_modal_level (CUDA, FP64)"})
    return ModalTimeSeriesResult(times.copy(), eta_total, comps, modal_audit)


def reconstruct_unidirectional_timeseries(eta1, time, *, depth: float, gravity: float = 9.81,
                                          omega_max: float | None = None,
                                          energy_fraction: float = 0.999, quadrature_rank: int = 8,
                                          order: int = 3,
                                          modal_points=(2048, 4096, 8192, 16384, 32768, 65536),
                                          modal_limit: float | None = None,
                                          relative_tolerance: float = 1.0e-3,
                                          include_eta20: bool = True, eta20_rank: int = 16,
                                          eta20_grid: tuple[int, int] = (128, 16), device=None,
                                          **unknown: Any) -> TimeSeriesResult:
    """The reference's default time interface (``temporal.py:19-60``)."""
    if unknown:
        raise TypeError(f"unknown time-reconstruction options: {', '.join(sorted(unknown))}")
    return reconstruct_unidirectional_modal_timeseries(
        eta1, time, depth=depth, gravity=gravity, omega_max=omega_max,
        energy_fraction=energy_fraction, quadrature_rank=quadrature_rank, order=order,
        modal_points=modal_points, modal_limit=modal_limit, relative_tolerance=relative_tolerance,
        include_eta20=include_eta20, eta20_rank=eta20_rank, eta20_grid=eta20_grid, device=device)
