"""Gradient of the GL surface elevation with respect to the first-order
amplitudes: a ``torch.autograd.Function`` over the engine's forward
(``gl_execute``) and reverse (``gl_adjoint_execute``) passes.

The reference evaluates the surface ``eta = eta11 + eta22 + eta33`` from the
first-order components ``a, b`` (``src/gl_spectral_coefficients.m`` ->
``src/gl_spectral_surface.m``); it has no gradient.  Here the surface is a
differentiable function of ``a, b`` so that a phase-resolved first-order
field can be fitted to an observed nonlinear surface::

    model = EtaSurfaceModel(kx, ky, depth=25.0, lx=512.0, ly=512.0, nx=512, ny=512)
    a = torch.tensor(a0, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    loss = ((eta_surface(a, b, model) - eta_obs) ** 2).sum()
    loss.backward()          # a.grad, b.grad from one adjoint pass

The backward pass stores nothing from the forward call: it re-deposits the
spectrum and re-evaluates, node by node, the forward fields each transposed
stage needs (the supports, balance shifts, scales, peak and roundoff-floor
decisions are those of the current ``a, b``, i.e. the derivative is the one
of the piecewise-polynomial map on its current piece).
"""

from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
import torch

from . import _lib, api


class EtaSurfaceModel:
    """Fixed geometry of a fit: modes (kx, ky), grid, depth, snapshot times.

    ``components`` picks the eta components summed into the surface (default:
    every eta component of ``order``: eta11, eta22, eta33).
    """

    def __init__(self, kx, ky, *, depth: float, lx: float, ly: float, nx: int, ny: int,
                 times=(0.0,), order: int = 3, gravity: float = 9.81, eta22_rank: int = 6,
                 order3_ranks=(4, 4), components: Sequence[str] | None = None,
                 grid: str = "compact", device=None, allow_below: bool = False):
        kx = np.asarray(kx, dtype=np.float64).ravel()
        ky = np.asarray(ky, dtype=np.float64).ravel()
        ones = np.ones_like(kx)
        coeffs = api.gl_spectral_coefficients(order, gravity, depth, ones, 0.0 * ones, kx, ky, 0.0,
                                              0.0, {"eta22_rank": eta22_rank,
                                                    "allow_below_model_parent_domain": allow_below})
        if components is None:
            components = [c for c in ("eta11", "eta22", "eta33")
                          if int(c[-1]) <= order]
        if any(not c.startswith("eta") for c in components):
            raise api.GLError("green_laplace:Options", "the surface gradient covers eta components only")
        self.components = tuple(components)
        self.times = np.atleast_1d(np.asarray(times, dtype=np.float64))
        self.n_times = int(self.times.size)
        self.nx, self.ny = int(nx), int(ny)
        self.n_modes = int(kx.size)
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise api.GLError("green_laplace:Device", "the GL engine runs on CUDA devices only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        dep = api.prepare_deposit(coeffs, lx, ly, self.nx, self.ny)
        self.deposit = dep
        mask = api._components_for(order, self.components)
        self.plan = api.get_plan(nx=self.nx, ny=self.ny, lx=float(lx), ly=float(ly), depth=float(depth),
                                 gravity=float(gravity), order=order, components=mask,
                                 eta22_rank=int(eta22_rank), allow_below=allow_below, box=dep.box,
                                 grid=api.GRID_REFERENCE if grid == "reference" else api.GRID_COMPACT,
                                 max_units=self.n_times, output=api.OUT_REAL, device=self.device,
                                 inner_rank=int(order3_ranks[0]), outer_rank=int(order3_ranks[1]))
        lib = _lib.load()
        size = C.c_size_t()
        api._engine_call(lib.gl_adjoint_workspace_size(self.plan.handle, C.byref(size)))
        self.adjoint_workspace_bytes = int(size.value)
        dev = self.device
        with torch.cuda.device(dev):
            t = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x)).to(dev, dt)  # noqa: E731
            self._seg_off = t(dep.seg_offsets, torch.int32)
            self._seg_bin = t(dep.seg_bins, torch.int32)
            self._omega = t(dep.omega, torch.float64)
            self._times = t(self.times, torch.float64)
            self._index = t(dep.index, torch.int64)
            self._adj_ws = torch.empty(self.adjoint_workspace_bytes + 256, dtype=torch.uint8, device=dev)
        w, h = dep.box[2], dep.box[3]
        self.box_shape = (h, w)

    # -- device passes -------------------------------------------------------

    def _spectra(self, a: torch.Tensor, b: torch.Tensor, stream: int) -> torch.Tensor:
        ab = torch.stack((a[self._index], b[self._index]), dim=1).contiguous()
        h, w = self.box_shape
        spec = torch.empty((self.n_times, h, w, 2), dtype=torch.float64, device=self.device)
        self.plan.deposit(self.n_times, self._seg_off, self._seg_bin, ab, self._omega, self._times,
                          spec, stream)
        return spec

    def _check_ab(self, a: torch.Tensor, b: torch.Tensor) -> None:
        for name, v in (("a", a), ("b", b)):
            if v.dtype != torch.float64 or v.device != self.device or v.shape != (self.n_modes,):
                raise api.GLError("green_laplace:ComponentSize",
                                  f"{name} must be a float64 tensor of shape ({self.n_modes},) on {self.device}")

    def eta(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        """Surface [time][ny][nx] (float64, metres) = sum of the model's eta components."""
        self._check_ab(a, b)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            spec = self._spectra(a.detach(), b.detach(), stream)
            ncomp = self.plan.info.n_components
            out = torch.empty((self.n_times, ncomp, self.ny, self.nx), dtype=torch.float64,
                              device=self.device)
            status = torch.zeros(self.n_times, dtype=torch.int32, device=self.device)
            self.plan.execute(self.n_times, spec, api.SPECTRA_BOX, out, status, stream)
            api._check_status(status)
            return out.sum(dim=1) if ncomp > 1 else out[:, 0]

    def vjp(self, a: torch.Tensor, b: torch.Tensor, grad_eta: torch.Tensor):
        """(dL/da, dL/db) for dL/deta = grad_eta ([time][ny][nx] or [ny][nx])."""
        self._check_ab(a, b)
        r = grad_eta.detach().to(device=self.device, dtype=torch.float64)
        r = r.reshape(self.n_times, self.ny, self.nx).contiguous()
        lib = _lib.load()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            spec = self._spectra(a.detach(), b.detach(), stream)
            h, w = self.box_shape
            g = torch.empty((self.n_times, h, w, 2), dtype=torch.float64, device=self.device)
            status = torch.zeros(self.n_times, dtype=torch.int32, device=self.device)
            ws = (self._adj_ws.data_ptr() + 255) & ~255
            api._engine_call(lib.gl_adjoint_execute(
                self.plan.handle, self.n_times, C.c_void_p(spec.data_ptr()), api.SPECTRA_BOX,
                C.c_void_p(r.data_ptr()), C.c_void_p(g.data_ptr()), C.c_void_p(ws),
                C.c_size_t(self.adjoint_workspace_bytes), C.c_void_p(status.data_ptr()),
                C.c_void_p(stream)))
            n_sel = int(self._index.numel())
            gab = torch.empty((n_sel, 2), dtype=torch.float64, device=self.device)
            api._engine_call(lib.gl_deposit_modes_adjoint(
                self.plan.handle, self.n_times, int(self._seg_bin.numel()),
                C.c_void_p(self._seg_off.data_ptr()), C.c_void_p(self._seg_bin.data_ptr()), n_sel,
                C.c_void_p(self._omega.data_ptr()), C.c_void_p(self._times.data_ptr()),
                C.c_void_p(g.data_ptr()), C.c_void_p(gab.data_ptr()), C.c_void_p(stream)))
            api._check_status(status)
            ga = torch.zeros(self.n_modes, dtype=torch.float64, device=self.device)
            gb = torch.zeros(self.n_modes, dtype=torch.float64, device=self.device)
            ga[self._index] = gab[:, 0]
            gb[self._index] = gab[:, 1]
        return ga, gb


class GLEtaSurface(torch.autograd.Function):
    """eta(a, b) through the engine; backward = one adjoint pass."""

    @staticmethod
    def forward(ctx, a, b, model: EtaSurfaceModel):
        ctx.model = model
        ctx.save_for_backward(a, b)
        return model.eta(a, b)

    @staticmethod
    def backward(ctx, grad_eta):
        a, b = ctx.saved_tensors
        ga, gb = ctx.model.vjp(a, b, grad_eta)
        return ga, gb, None


def eta_surface(a: torch.Tensor, b: torch.Tensor, model: EtaSurfaceModel) -> torch.Tensor:
    """Differentiable GL surface [time][ny][nx] for first-order amplitudes a, b."""
    return GLEtaSurface.apply(a, b, model)
