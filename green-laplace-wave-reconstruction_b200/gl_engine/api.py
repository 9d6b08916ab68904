"""Reference-facing Python API of the B200 Green--Laplace engine.

Mirrors the reference's calling patterns:

* MATLAB two-stage API -- ``gl_spectral_coefficients(order, g, h, a, b, kx,
  ky, Ux, Uy, options)`` (``src/gl_spectral_coefficients.m:1-112``) then
  ``gl_spectral_surface(coeffs, Lx, Ly, Nx, Ny, t)`` returning
  ``(eta, psi, X, Y, components, audit)`` (``src/gl_spectral_surface.m:1-103``);
* Python package API -- ``reconstruct_directional_field(eta1, *, lx, ly,
  depth, gravity, time, order, eta22_rank, allow_below_model_parent_domain)``
  (``python/src/green_laplace/spatial.py:33-153``).

Validation errors raise :class:`GLError` (a ``ValueError``) carrying the
MATLAB identifier (``green_laplace:<Id>``).  All GL arithmetic runs in the
native CUDA library through its C ABI; nothing here computes a field on the
CPU.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Any, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import (COMP_ETA11, COMP_ETA22, COMP_ETA33, COMP_NAMES, COMP_PSI11, COMP_PSI22,
                   COMP_PSI33, GRID_COMPACT, GRID_REFERENCE, OUT_COMPLEX, OUT_REAL, SPECTRA_BOX,
                   SPECTRA_FULL, PlanDesc, PlanInfo)

API_NAME = "green-laplace-spectral-v1"


class GLError(ValueError):
    """Validation error with the reference's MATLAB identifier."""

    def __init__(self, identifier: str, message: str):
        super().__init__(message)
        self.identifier = identifier


# gl_status -> (MATLAB identifier, message) for per-unit device statuses
_STATUS_ERRORS = {
    6: ("green_laplace:Components", "Component amplitudes and nonzero wavenumbers must be finite."),
    10: ("green_laplace:Order2Domain", "psi22 requires parent kh >= 0.3"),
    11: ("green_laplace:Order3Domain",
         "third-order reconstruction requires strict-forward parent kh > 0.5"),
    15: ("green_laplace:Scale", "invalid Green--Laplace scale"),
    17: ("green_laplace:Support", "eta1 has empty analytic support"),
    18: ("green_laplace:Support", "spectrum support lies outside the plan's parent box"),
    19: ("green_laplace:NonFinite", "non-finite value in a reconstructed field"),
}


def _status_error(code: int) -> GLError:
    ident, msg = _STATUS_ERRORS.get(code, ("green_laplace:Engine", f"engine status {code}"))
    return GLError(ident, msg)


def _engine_call(status: int) -> None:
    if status != 0:
        msg = _lib.last_error()
        ident = {
            2: "green_laplace:Unsupported", 13: "green_laplace:Nyquist",
            14: "green_laplace:Nyquist", 7: "green_laplace:Support", 16: "green_laplace:Rank",
        }.get(status)
        if ident is not None:
            raise GLError(ident, msg)
        raise _lib.EngineError(status, msg)


# ---------------------------------------------------------------------------
# stage 1: coefficients (gl_spectral_coefficients.m)
# ---------------------------------------------------------------------------

_DEFAULT_OPTIONS = {
    "sector": "pure-sum",
    "eta22_rank": 6,
    "peak_wavenumber": None,
    "allow_below_model_parent_domain": False,
    "grid_tolerance": 1e-10,
}


@dataclass(frozen=True)
class GLCoefficients:
    """Output of :func:`gl_spectral_coefficients` (fields of ``gl_spectral_coefficients.m:74-87``)."""

    order: int
    g: float
    h: float
    a: np.ndarray
    b: np.ndarray
    kx: np.ndarray
    ky: np.ndarray
    Ux: float
    Uy: float
    intrinsic_omega: np.ndarray
    omega: np.ndarray
    peak_wavenumber: float
    peak_depth: float
    options: dict = field(default_factory=dict)
    api: str = API_NAME
    information_boundary: str = "first-order surface elevation only"
    surface_potential_definition: str = "psi=phi(x,z=eta,t)"
    flat_potential_is_public_output: bool = False


def gl_spectral_coefficients(order, g, h, a, b, kx, ky, Ux=0.0, Uy=0.0, options=None
                             ) -> GLCoefficients:
    """Validate first-order components and prepare a GL reconstruction.

    Restates the checks of ``src/gl_spectral_coefficients.m:6-71`` with the
    same identifiers.
    """
    opts = dict(_DEFAULT_OPTIONS)
    if options is not None:
        if not isinstance(options, dict):
            raise GLError("green_laplace:Options", "The optional input must be one options struct.")
        for key, value in options.items():
            if key not in opts:
                raise GLError("green_laplace:UnknownOption", f"Unknown Green--Laplace option: {key}")
            opts[key] = value
    opts["sector"] = str(opts["sector"])
    opts["allow_below_model_parent_domain"] = bool(opts["allow_below_model_parent_domain"])
    if not (isinstance(order, (int, np.integer)) and 1 <= int(order) <= 3):
        raise GLError("green_laplace:Order", "order must be an integer from 1 to 3")
    for name, value in (("g", g), ("h", h)):
        if not (np.isscalar(value) and np.isfinite(value) and value > 0):
            raise GLError("green_laplace:Scalar", f"{name} must be a finite positive scalar")
    for name, value in (("Ux", Ux), ("Uy", Uy)):
        if not (np.isscalar(value) and np.isfinite(value)):
            raise GLError("green_laplace:Scalar", f"{name} must be a finite scalar")
    if Ux != 0 or Uy != 0:
        raise GLError("green_laplace:UniformCurrent",
                      "The released API preserves the MF12-compatible Ux, Uy input slots "
                      "but has only been certified for Ux=Uy=0.")
    a, b, kx, ky = (np.asarray(v, dtype=float).ravel() for v in (a, b, kx, ky))
    if a.size == 0 or not (a.size == b.size == kx.size == ky.size):
        raise GLError("green_laplace:ComponentSize",
                      "a, b, kx, and ky must be nonempty vectors of equal length.")
    if not np.all(np.isfinite(np.concatenate([a, b, kx, ky]))) or np.any(np.hypot(kx, ky) <= 0):
        raise GLError("green_laplace:Components",
                      "Component amplitudes and nonzero wavenumbers must be finite.")
    if np.any(kx <= 0):
        raise GLError("green_laplace:Support",
                      "The released GL graphs require strict-forward support kx>0.")
    if opts["sector"] != "pure-sum":
        raise GLError("green_laplace:Sector",
                      "The released total-field API supports the positive pure-sum sector only.")
    rank = opts["eta22_rank"]
    if not (isinstance(rank, (int, np.integer)) and 1 <= int(rank) <= 12):
        raise GLError("green_laplace:Rank", "eta22_rank must be a positive integer <= 12")
    amp = np.hypot(a, b)
    if not np.any(amp > 0):
        raise GLError("green_laplace:ZeroInput", "At least one input amplitude is required.")
    k = np.hypot(kx, ky)
    if opts["peak_wavenumber"] is None:
        peak_k = float(k[int(np.argmax(amp**2))])
    else:
        pk = opts["peak_wavenumber"]
        if not (np.isscalar(pk) and np.isfinite(pk) and pk > 0):
            raise GLError("green_laplace:Options", "peak_wavenumber must be a finite positive scalar")
        peak_k = float(pk)
    parent_q = h * k
    if order >= 2 and np.any(parent_q < 0.3) and not opts["allow_below_model_parent_domain"]:
        raise GLError("green_laplace:Order2Domain",
                      "Order-two surface-potential reconstruction requires kh>=0.3. "
                      "A labelled tail extrapolation can be enabled in options.")
    if order >= 3 and np.any(parent_q <= 0.5):
        raise GLError("green_laplace:Order3Domain",
                      "Order-three reconstruction requires every parent kh>0.5.")
    intrinsic = np.sqrt(g * k * np.tanh(h * k))
    return GLCoefficients(order=int(order), g=float(g), h=float(h), a=a, b=b, kx=kx, ky=ky,
                          Ux=float(Ux), Uy=float(Uy), intrinsic_omega=intrinsic,
                          omega=kx * Ux + ky * Uy + intrinsic, peak_wavenumber=peak_k,
                          peak_depth=float(h * peak_k), options=opts)


# ---------------------------------------------------------------------------
# plans and device execution
# ---------------------------------------------------------------------------


class Plan:
    """An engine plan plus its device workspace on one CUDA device."""

    def __init__(self, desc: PlanDesc, device: torch.device):
        self.lib = _lib.load()
        self.device = device
        self.desc = desc
        with torch.cuda.device(device):
            handle = C.c_void_p()
            _engine_call(self.lib.gl_plan_create(C.byref(handle), C.byref(desc)))
            self.handle = handle
            info = PlanInfo()
            _engine_call(self.lib.gl_plan_get_info(handle, C.byref(info)))
            self.info = info
            size = C.c_size_t()
            _engine_call(self.lib.gl_workspace_size(handle, C.byref(size)))
            self.workspace_bytes = int(size.value)
            self._workspace = None
            self._retired: list[torch.Tensor] = []
            self.lanes = 1

    @property
    def workspace(self) -> torch.Tensor:
        """Device workspace, allocated on first use (batches pass a shared one)."""
        if self._workspace is None:
            self._workspace = torch.empty(max(self.workspace_bytes, 256) + 256, dtype=torch.uint8,
                                          device=self.device)
        return self._workspace

    @property
    def component_ids(self) -> list[int]:
        return [self.info.component_ids[i] for i in range(self.info.n_components)]

    @property
    def box(self) -> tuple[int, int, int, int]:
        return tuple(self.info.box1)

    def set_tuning(self, pair_row_groups: int = 0, triple_row_groups: int = 0,
                   col_block_columns: int = 0) -> None:
        """Launch shapes of this plan's transform kernels (0: built-in choice)."""
        t = _lib.Tuning(pair_row_groups, triple_row_groups, col_block_columns)
        _engine_call(self.lib.gl_plan_set_tuning(self.handle, C.byref(t)))
        self.tuning = (pair_row_groups, triple_row_groups, col_block_columns)

    def set_lanes(self, lanes: int) -> None:
        """Run this plan's unit groups on ``lanes`` concurrent streams
        (``gl_plan_set_lanes``): groups of ceil(max_units / lanes) units, group
        i on lane i mod lanes, bitwise the same outputs.  Re-sizes the
        workspace."""
        with torch.cuda.device(self.device):
            _engine_call(self.lib.gl_plan_set_lanes(self.handle, int(lanes)))
            size = C.c_size_t()
            _engine_call(self.lib.gl_workspace_size(self.handle, C.byref(size)))
        self.workspace_bytes = int(size.value)
        if self._workspace is not None:
            # graphs captured before this call keep launching into the old
            # workspace with the old layout: keep it alive with the plan
            self._retired.append(self._workspace)
        self._workspace = None
        self.lanes = min(int(lanes), int(self.desc.max_units))

    def _ws_ptr(self) -> int:
        ptr = self.workspace.data_ptr()
        return (ptr + 255) & ~255

    def deposit(self, n_units: int, seg_offsets: torch.Tensor, seg_bins: torch.Tensor,
                ab: torch.Tensor, omega: torch.Tensor, times: torch.Tensor, out: torch.Tensor,
                stream: int) -> None:
        _engine_call(self.lib.gl_deposit_modes(
            self.handle, n_units, int(seg_bins.numel()), C.c_void_p(seg_offsets.data_ptr()),
            C.c_void_p(seg_bins.data_ptr()), int(omega.numel()), C.c_void_p(ab.data_ptr()),
            C.c_void_p(omega.data_ptr()), C.c_void_p(times.data_ptr()),
            C.c_void_p(out.data_ptr()), C.c_void_p(stream)))

    def execute(self, n_units: int, spectra: torch.Tensor, layout: int, out: torch.Tensor,
                status: torch.Tensor | None, stream: int) -> None:
        _engine_call(self.lib.gl_execute(
            self.handle, n_units, C.c_void_p(spectra.data_ptr()), layout,
            C.c_void_p(out.data_ptr()), C.c_void_p(self._ws_ptr()),
            C.c_size_t(self.workspace_bytes),
            C.c_void_p(status.data_ptr()) if status is not None else None, C.c_void_p(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                self.lib.gl_plan_destroy(self.handle)
        except Exception:
            pass


_PLANS: dict[tuple, Plan] = {}


def get_plan(*, nx, ny, lx, ly, depth, gravity, order, components, eta22_rank, allow_below,
             box, grid, max_units, output, device, inner_rank=4, outer_rank=4) -> Plan:
    key = (nx, ny, float(lx), float(ly), float(depth), float(gravity), order, components,
           eta22_rank, bool(allow_below), tuple(box), grid, max_units, output, str(device),
           inner_rank, outer_rank)
    plan = _PLANS.get(key)
    if plan is None:
        desc = PlanDesc(nx=nx, ny=ny, lx=lx, ly=ly, depth=depth, gravity=gravity, order=order,
                        components=components, eta22_rank=eta22_rank, inner_rank=inner_rank,
                        outer_rank=outer_rank,
                        allow_below_model_parent_domain=int(bool(allow_below)),
                        box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3], grid=grid,
                        max_units=max_units, output=output)
        plan = Plan(desc, device)
        if len(_PLANS) > 64:
            _PLANS.clear()
        _PLANS[key] = plan
    return plan


def _matlab_round(v: np.ndarray) -> np.ndarray:
    return np.sign(v) * np.floor(np.abs(v) + 0.5)


@dataclass
class ModeDeposit:
    """Host-side deposit bookkeeping for one set of modes on one grid."""

    box: tuple[int, int, int, int]
    seg_offsets: np.ndarray
    seg_bins: np.ndarray
    ab: np.ndarray
    omega: np.ndarray
    index: np.ndarray | None = None   # deposit order -> input mode index


def prepare_deposit(coeffs: GLCoefficients, lx, ly, nx, ny) -> ModeDeposit:
    """Mode -> bin mapping with the off-grid and Nyquist checks of
    ``deposit_analytic_input`` (``src/gl_spectral_surface.m:123-149``)."""
    dkx = 2.0 * np.pi / lx
    dky = 2.0 * np.pi / ly
    mx = _matlab_round(coeffs.kx / dkx)
    my = _matlab_round(coeffs.ky / dky)
    tol = coeffs.options["grid_tolerance"] * np.maximum(1.0, np.hypot(coeffs.kx, coeffs.ky))
    if np.any(np.abs(coeffs.kx - mx * dkx) > tol) or np.any(np.abs(coeffs.ky - my * dky) > tol):
        raise GLError("green_laplace:OffGridComponent",
                      "Every component must lie on the requested FFT grid.")
    if np.any(np.abs(mx) >= nx / 2) or np.any(np.abs(my) >= ny / 2):
        raise GLError("green_laplace:Nyquist",
                      "An input component reaches or exceeds a Nyquist boundary.")
    mx = mx.astype(np.int64)
    my = my.astype(np.int64)
    live = np.hypot(coeffs.a, coeffs.b) > 0
    idx = np.flatnonzero(live)
    x0, x1 = int(mx[idx].min()), int(mx[idx].max())
    y0, y1 = int(my[idx].min()), int(my[idx].max())
    box = (x0, y0, x1 - x0 + 1, y1 - y0 + 1)
    bins = (my[idx] - y0) * box[2] + (mx[idx] - x0)
    order = np.argsort(bins, kind="stable")
    sb = bins[order]
    starts = np.flatnonzero(np.r_[True, sb[1:] != sb[:-1]])
    seg_offsets = np.r_[starts, sb.size].astype(np.int32)
    seg_bins = sb[starts].astype(np.int32)
    sel = idx[order]
    ab = np.stack([coeffs.a[sel], coeffs.b[sel]], axis=1).astype(np.float64).ravel()
    return ModeDeposit(box=box, seg_offsets=seg_offsets, seg_bins=seg_bins, ab=ab,
                       omega=coeffs.omega[sel].astype(np.float64), index=sel.astype(np.int64))


def _components_for(order: int, components: Sequence[str] | None) -> int:
    if components is None:
        mask = COMP_ETA11 | COMP_PSI11
        if order >= 2:
            mask |= COMP_ETA22 | COMP_PSI22
        if order >= 3:
            mask |= COMP_ETA33 | COMP_PSI33
        return mask
    inv = {v: k for k, v in COMP_NAMES.items()}
    mask = 0
    for name in components:
        if name not in inv:
            raise GLError("green_laplace:Options", f"unknown component {name!r}")
        mask |= inv[name]
    return mask


@dataclass
class SurfaceBatch:
    """Device-resident result of a batched surface evaluation."""

    fields: torch.Tensor            # [unit][component][ny][nx]
    names: list[str]
    status: torch.Tensor            # [unit] gl_status
    plan: Plan

    def component(self, name: str) -> torch.Tensor:
        return self.fields[:, self.names.index(name)]


def _check_status(status: torch.Tensor) -> None:
    host = status.cpu().numpy()
    bad = np.flatnonzero(host != 0)
    if bad.size:
        raise _status_error(int(host[bad[0]]))


def surface_batch_device(coeffs: GLCoefficients, Lx, Ly, Nx, Ny, times, *,
                         components: Sequence[str] | None = None, output: str = "complex",
                         grid: str = "compact", device=None, max_units: int | None = None,
                         check: bool = True, stream: torch.cuda.Stream | None = None,
                         out: torch.Tensor | None = None, order3_ranks=(4, 4)) -> SurfaceBatch:
    """Evaluate ``len(times)`` snapshots of one sea state on the GPU.

    Inputs are host arrays; outputs stay on the device.  ``components``
    selects a subset of eta11..psi33 (default: all of the coefficients' order);
    ``order3_ranks`` = (inner, outer) GL ranks of the order-3 graph (the
    reference's unified API fixes GL4/GL4, ``_order3.py:23-26``).
    """
    if not isinstance(coeffs, GLCoefficients) or coeffs.api != API_NAME:
        raise GLError("green_laplace:Coefficients", "Input must come from gl_spectral_coefficients.")
    for name, value in (("Lx", Lx), ("Ly", Ly)):
        if not (np.isscalar(value) and np.isfinite(value) and value > 0):
            raise GLError("green_laplace:Grid", f"{name} must be a finite positive scalar")
    for name, value in (("Nx", Nx), ("Ny", Ny)):
        if not (isinstance(value, (int, np.integer)) and value > 0 and value % 2 == 0):
            raise GLError("green_laplace:Grid", f"{name} must be a positive even integer")
    times = np.atleast_1d(np.asarray(times, dtype=np.float64))
    if not np.all(np.isfinite(times)):
        raise GLError("green_laplace:Grid", "t must be finite")
    device = torch.device(device if device is not None else "cuda")
    if device.type != "cuda":
        raise GLError("green_laplace:Device", "the GL engine runs on CUDA devices only")
    mask = _components_for(coeffs.order, components)
    dep = prepare_deposit(coeffs, Lx, Ly, int(Nx), int(Ny))
    n = int(times.size)
    out_mode = OUT_REAL if output == "real" else OUT_COMPLEX
    plan = get_plan(nx=int(Nx), ny=int(Ny), lx=float(Lx), ly=float(Ly), depth=coeffs.h,
                    gravity=coeffs.g, order=coeffs.order, components=mask,
                    eta22_rank=int(coeffs.options["eta22_rank"]),
                    allow_below=coeffs.options["allow_below_model_parent_domain"], box=dep.box,
                    grid=GRID_REFERENCE if grid == "reference" else GRID_COMPACT,
                    max_units=max_units or min(n, 8), output=out_mode, device=device,
                    inner_rank=int(order3_ranks[0]), outer_rank=int(order3_ranks[1]))
    stream = stream or torch.cuda.current_stream(device)
    with torch.cuda.device(device), torch.cuda.stream(stream):
        def h2d(arr, dtype):
            # staged through pinned memory so the copy is asynchronous (a
            # pageable source would synchronise the stream first)
            host = torch.from_numpy(np.ascontiguousarray(arr)).to(dtype=dtype).pin_memory()
            return host.to(device=device, non_blocking=True)
        seg_off = h2d(dep.seg_offsets, torch.int32)
        seg_bin = h2d(dep.seg_bins, torch.int32)
        ab = h2d(dep.ab, torch.float64)
        om = h2d(dep.omega, torch.float64)
        tt = h2d(times, torch.float64)
        w, h = dep.box[2], dep.box[3]
        box_spec = torch.empty((n, h, w, 2), dtype=torch.float64, device=device)
        plan.deposit(n, seg_off, seg_bin, ab, om, tt, box_spec, stream.cuda_stream)
        ncomp = plan.info.n_components
        dtype = torch.float64 if out_mode == OUT_REAL else torch.complex128
        if out is None:
            out = torch.empty((n, ncomp, int(Ny), int(Nx)), dtype=dtype, device=device)
        status = torch.zeros(n, dtype=torch.int32, device=device)
        plan.execute(n, box_spec, SPECTRA_BOX, out, status, stream.cuda_stream)
    names = [COMP_NAMES[c] for c in plan.component_ids]
    res = SurfaceBatch(fields=out, names=names, status=status, plan=plan)
    if check:
        _check_status(status)
    return res


class SurfaceStream:
    """Batches of snapshots of one sea state streamed to pinned host memory.

    ``submit(times)`` evaluates one batch and queues the device->host copy of
    its fields on a separate copy stream, so the copy of batch i overlaps the
    evaluation of batch i+1.  ``result(ticket)`` waits for that batch's copy
    and returns its host fields; a host buffer is reused two submissions
    later, so read (or copy) a result before submitting twice more.

    Every batch copies its inputs -- the sea state's mode table and the batch's
    times -- from pinned host staging buffers to the device and runs the
    deposit and the whole engine graph.  The mode -> bin mapping is prepared
    on the host once per stream, and with ``graphs=True`` (the default) the
    per-batch work -- input copies, deposit, every engine launch -- is one
    captured CUDA graph per (buffer slot, batch size), replayed per batch, so
    the host spends microseconds instead of a launch sequence per batch.
    """

    def __init__(self, coeffs: GLCoefficients, Lx, Ly, Nx, Ny, *,
                 components: Sequence[str] | None = None, output: str = "real",
                 grid: str = "compact", device=None, max_units: int | None = None,
                 check: bool = True, order3_ranks=(4, 4), graphs: bool = True):
        self._args = (coeffs, Lx, Ly, Nx, Ny)
        self._kw = dict(components=components, output=output, grid=grid,
                        max_units=max_units, order3_ranks=order3_ranks)
        self.device = torch.device(device if device is not None else "cuda")
        self.check = check
        self.graphs = graphs
        self._copy = torch.cuda.Stream(self.device)
        self._host: list[torch.Tensor | None] = [None, None]
        self._computed = [torch.cuda.Event(), torch.cuda.Event()]
        self._copied = [torch.cuda.Event(), torch.cuda.Event()]
        self._names: list[str] = []
        self._plan: Plan | None = None
        self._submitted = 0
        self._dep = prepare_deposit(coeffs, Lx, Ly, int(Nx), int(Ny))
        self._slots: dict = {}  # (slot, n) -> staged buffers and graph
        self._cur: list[dict | None] = [None, None]  # the buffers of each slot's last batch

    def _stage(self, slot: int, n: int) -> dict:
        """Pinned staging buffers, device buffers and (optionally) the graph
        of one buffer slot and batch size."""
        key = (slot, n)
        if key in self._slots:
            return self._slots[key]
        coeffs, Lx, Ly, Nx, Ny = self._args
        kw = self._kw
        dep = self._dep
        dev = self.device
        mask = _components_for(coeffs.order, kw["components"])
        out_mode = OUT_REAL if kw["output"] == "real" else OUT_COMPLEX
        plan = get_plan(nx=int(Nx), ny=int(Ny), lx=float(Lx), ly=float(Ly), depth=coeffs.h,
                        gravity=coeffs.g, order=coeffs.order, components=mask,
                        eta22_rank=int(coeffs.options["eta22_rank"]),
                        allow_below=coeffs.options["allow_below_model_parent_domain"],
                        box=dep.box,
                        grid=GRID_REFERENCE if kw["grid"] == "reference" else GRID_COMPACT,
                        max_units=kw["max_units"] or min(n, 8), output=out_mode, device=dev,
                        inner_rank=int(kw["order3_ranks"][0]),
                        outer_rank=int(kw["order3_ranks"][1]))
        pin = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dt).pin_memory()  # noqa: E731
        st = {
            "plan": plan,
            "h_seg_off": pin(dep.seg_offsets, torch.int32),
            "h_seg_bin": pin(dep.seg_bins, torch.int32),
            "h_ab": pin(dep.ab, torch.float64),
            "h_om": pin(dep.omega, torch.float64),
            "h_t": torch.zeros(n, dtype=torch.float64).pin_memory(),
        }
        for k in ("seg_off", "seg_bin", "ab", "om", "t"):
            st["d_" + k] = torch.empty_like(st["h_" + k], device=dev)
        w, h = dep.box[2], dep.box[3]
        st["spec"] = torch.empty((n, h, w, 2), dtype=torch.float64, device=dev)
        dtype = torch.float64 if out_mode == OUT_REAL else torch.complex128
        st["out"] = torch.empty((n, plan.info.n_components, int(Ny), int(Nx)), dtype=dtype,
                                device=dev)
        st["status"] = torch.zeros(n, dtype=torch.int32, device=dev)
        st["graph"] = None
        self._slots[key] = st
        return st

    def _enqueue(self, st: dict, stream: torch.cuda.Stream) -> None:
        """Input copies from the pinned staging buffers, deposit, engine."""
        n = st["h_t"].numel()
        with torch.cuda.stream(stream):
            for k in ("seg_off", "seg_bin", "ab", "om", "t"):
                st["d_" + k].copy_(st["h_" + k], non_blocking=True)
            plan = st["plan"]
            plan.deposit(n, st["d_seg_off"], st["d_seg_bin"], st["d_ab"], st["d_om"], st["d_t"],
                         st["spec"], stream.cuda_stream)
            plan.execute(n, st["spec"], SPECTRA_BOX, st["out"], st["status"], stream.cuda_stream)

    def submit(self, times) -> int:
        slot = self._submitted % 2
        times = np.atleast_1d(np.asarray(times, dtype=np.float64))
        if not np.all(np.isfinite(times)):
            raise GLError("green_laplace:Grid", "t must be finite")
        n = int(times.size)
        comp = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            st = self._stage(slot, n)
            # the slot's previous evaluation has read its staging buffers and
            # its previous copy has read its fields
            self._copied[slot].synchronize()
            st["h_t"].numpy()[:] = times
            comp.wait_event(self._copied[slot])
            if self.graphs and st["graph"] is None:
                self._enqueue(st, comp)  # eager once: kernel attributes, caches
                comp.synchronize()
                g = torch.cuda.CUDAGraph()
                side = torch.cuda.Stream(self.device)
                side.wait_stream(comp)
                with torch.cuda.stream(side):
                    with torch.cuda.graph(g, stream=side):
                        self._enqueue(st, side)
                comp.wait_stream(side)
                st["graph"] = g
            if self.graphs:
                with torch.cuda.stream(comp):
                    st["graph"].replay()
            else:
                self._enqueue(st, comp)
        self._names = [COMP_NAMES[c] for c in st["plan"].component_ids]
        self._plan = st["plan"]
        self._cur[slot] = st
        self._computed[slot].record(comp)
        host = self._host[slot]
        if host is None or host.shape != st["out"].shape:
            host = torch.empty(st["out"].shape, dtype=st["out"].dtype, pin_memory=True)
            self._host[slot] = host
        self._copy.wait_event(self._computed[slot])
        with torch.cuda.stream(self._copy):
            host.copy_(st["out"], non_blocking=True)
        self._copied[slot].record(self._copy)
        self._submitted += 1
        return self._submitted - 1

    def result(self, ticket: int) -> SurfaceBatch:
        if not 0 <= ticket < self._submitted or ticket < self._submitted - 2:
            raise ValueError("ticket is not one of the last two submissions")
        slot = ticket % 2
        self._copied[slot].synchronize()
        st = self._cur[slot]
        if self.check:
            _check_status(st["status"])
        return SurfaceBatch(fields=self._host[slot], names=self._names, status=st["status"],
                            plan=self._plan)


def _audit(coeffs: GLCoefficients, plan: Plan, names, Lx, Ly, Nx, Ny, t) -> dict[str, Any]:
    info = plan.info
    comp_audits: dict[str, Any] = {}
    if coeffs.order >= 2:
        comp_audits["eta22"] = {"implementation": "prescribed-rank-green-laplace-eta22",
                                "quadrature_rank": int(coeffs.options["eta22_rank"]),
                                "candidate_id": "gl-eta22-pure-prescribed-rank-v1"}
        comp_audits["psi22"] = {"implementation": "dual-branch-green-laplace-psi22",
                                "quadrature_rank_total": 4,
                                "candidate_id": "gl-psi22-dual-branch-radial2-v1"}
    if coeffs.order >= 3:
        comp_audits["order3"] = {"implementation": "nested-no-stokes-green-laplace-order3",
                                 "inner_quadrature_rank": 4, "outer_quadrature_rank": 4,
                                 "candidate_id": "gl-eta33-psi33-stable-v1"}
    return {
        "api": coeffs.api,
        "order": coeffs.order,
        "sector": coeffs.options["sector"],
        "included_components": names,
        "surface_potential_definition": "psi=phi(x,z=eta,t)",
        "flat_potential_exposed": False,
        "rescaling_alignment_or_gain": False,
        "grid": [int(Ny), int(Nx)],
        "domain": [float(Ly), float(Lx)],
        "time": t,
        "component_audits": comp_audits,
        "engine": {
            "implementation": "gl-b200-cuda",
            "precision": "fp64",
            "product_grid": [info.ncy, info.ncx],
            "column_grids": {"pair": info.ncy_pair, "triple": info.ncy_triple},
            "pair_row_length": info.ncx_pair,
            "parent_box": list(info.box1),
            "reference_transforms_per_unit": info.transforms_per_unit,
        },
    }


def _xy(Lx, Ly, Nx, Ny):
    return np.meshgrid(np.arange(Nx) * (Lx / Nx), np.arange(Ny) * (Ly / Ny))


def gl_spectral_surface(coeffs: GLCoefficients, Lx, Ly, Nx, Ny, t, *, grid: str = "compact",
                        device=None):
    """Stage 2 of the two-stage API: ``(eta, psi, X, Y, components, audit)``.

    Mirrors ``src/gl_spectral_surface.m:1-103``; fields are numpy arrays.
    """
    res = surface_batch_device(coeffs, Lx, Ly, Nx, Ny, [t], grid=grid, device=device)
    fields = res.fields[0].cpu().numpy()
    components: dict[str, np.ndarray] = {}
    eta_plus = np.zeros((int(Ny), int(Nx)), dtype=complex)
    psi_plus = np.zeros_like(eta_plus)
    for k, name in enumerate(res.names):
        components[name + "_plus"] = fields[k]
        components[name] = np.real(fields[k])
        if name.startswith("eta"):
            eta_plus += fields[k]
        else:
            psi_plus += fields[k]
    components["eta_plus"] = eta_plus
    components["psi_plus"] = psi_plus
    components["eta"] = np.real(eta_plus)
    components["psi"] = np.real(psi_plus)
    X, Y = _xy(Lx, Ly, int(Nx), int(Ny))
    audit = _audit(coeffs, res.plan, res.names, Lx, Ly, Nx, Ny, float(t))
    return components["eta"], components["psi"], X, Y, components, audit


# ---------------------------------------------------------------------------
# Python-package entry: a real eta1 grid
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class DirectionalFieldResult:
    """Fields and execution information (``spatial.py:21-30``)."""

    x: np.ndarray
    y: np.ndarray
    eta: np.ndarray
    psi: np.ndarray
    components: dict
    audit: dict


def fft2_device(x: torch.Tensor, inverse: bool = False) -> torch.Tensor:
    """numpy-convention fft2/ifft2 of a [..., ny, nx] complex128 CUDA tensor (native kernels)."""
    lib = _lib.load()
    x = x.contiguous()
    ny, nx = x.shape[-2], x.shape[-1]
    batch = int(x.numel() // (nx * ny))
    out = torch.empty_like(x)
    with torch.cuda.device(x.device):
        _engine_call(lib.gl_fft2(batch, nx, ny, C.c_void_p(x.data_ptr()),
                                 C.c_void_p(out.data_ptr()), int(inverse),
                                 C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)))
    return out


def reconstruct_directional_field(eta1, *, lx: float, ly: float, depth: float,
                                  gravity: float = 9.81, time: float = 0.0, order: int = 2,
                                  eta22_rank: int = 6, allow_below_model_parent_domain: bool = False,
                                  device=None, grid: str = "compact") -> DirectionalFieldResult:
    """Strict-forward directional reconstruction from a real ``eta1`` grid
    (``python/src/green_laplace/spatial.py:33-153``)."""
    field_ = np.asarray(eta1, dtype=float)
    if field_.ndim != 2:
        raise ValueError("eta1 must be a two-dimensional array")
    if not np.isfinite(time) or depth <= 0 or gravity <= 0:
        raise ValueError("time must be finite; depth and gravity must be positive")
    if order not in (1, 2, 3):
        raise ValueError("order must be 1, 2, or 3")
    if not isinstance(eta22_rank, int) or eta22_rank < 1 or eta22_rank > 16:
        raise ValueError("eta22_rank must be an integer from 1 to 16")
    ny, nx = field_.shape
    if lx <= 0 or ly <= 0 or nx < 2 or ny < 2 or nx % 2 or ny % 2:
        raise ValueError("positive domain lengths and positive even grid sizes are required")
    if not np.all(np.isfinite(field_)):
        raise ValueError("eta1 must be a finite two-dimensional grid")
    dev = torch.device(device if device is not None else "cuda")
    tol = 1.0e-11
    with torch.cuda.device(dev):
        e1 = torch.from_numpy(field_).to(dev)
        raw = fft2_device((e1 / depth).to(torch.complex128))
        mag = raw.abs()
        scale = max(float(mag.max()), np.finfo(float).tiny)
        # kx == 0 column (_spectral.py:31-33)
        if float(mag[:, 0].max()) > tol * scale:
            raise ValueError("eta1 contains a non-negligible kx=0 component")
        spec = torch.zeros_like(raw)
        spec[:, 1:nx // 2] = 2.0 * raw[:, 1:nx // 2]
        rec = torch.real(depth * fft2_device(spec, inverse=True))
        err = float(torch.linalg.norm(rec - e1) / max(float(torch.linalg.norm(e1)),
                                                      np.finfo(float).tiny))
        if err > tol:
            raise ValueError("eta1 is not consistent with the declared strict-forward x propagation")
        # time phase exp(-i sqrt(g/h) nu t) (spatial.py:67-72)
        kx_line = 2.0 * np.pi * np.fft.fftfreq(nx, d=lx / nx)
        ky_line = 2.0 * np.pi * np.fft.fftfreq(ny, d=ly / ny)
        kxg, kyg = np.meshgrid(kx_line, ky_line)
        q = np.hypot(depth * kxg, depth * kyg)
        nu = np.sqrt(q * np.tanh(q))
        if time != 0.0:
            phase = torch.from_numpy(np.exp(-1j * np.sqrt(gravity / depth) * nu * time)).to(dev)
            spec = spec * phase
        amag = spec.abs()
        thr = 1.0e-13 * max(1.0, float(amag.max()))
        sup = amag > thr
        if not bool(sup.any()):
            raise ValueError("eta1 has empty analytic support")
        rows = torch.nonzero(sup.any(dim=1)).flatten().cpu().numpy()
        cols = torch.nonzero(sup.any(dim=0)).flatten().cpu().numpy()
        mys = np.where(rows < ny // 2, rows, rows - ny)
        mxs = np.where(cols < nx // 2, cols, cols - nx)
        if np.any(mxs <= 0):
            raise ValueError("strict-forward nonzero analytic eta1 support is required")
        box = (int(mxs.min()), int(mys.min()), int(mxs.max() - mxs.min() + 1),
               int(mys.max() - mys.min() + 1))
        mask = _components_for(order, None)
        try:
            plan = get_plan(nx=nx, ny=ny, lx=float(lx), ly=float(ly), depth=float(depth),
                            gravity=float(gravity), order=order, components=mask,
                            eta22_rank=eta22_rank, allow_below=allow_below_model_parent_domain,
                            box=box, grid=GRID_REFERENCE if grid == "reference" else GRID_COMPACT,
                            max_units=1, output=OUT_COMPLEX, device=dev)
        except GLError as exc:
            if exc.identifier == "green_laplace:Nyquist" and order >= 2:
                kind = "cubic" if order >= 3 else "quadratic"
                raise ValueError(f"{kind} output support reaches a Nyquist boundary") from exc
            raise
        out = torch.empty((1, plan.info.n_components, ny, nx), dtype=torch.complex128, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        plan.execute(1, torch.view_as_real(spec.contiguous()), SPECTRA_FULL, out, status,
                     torch.cuda.current_stream(dev).cuda_stream)
        code = int(status.cpu()[0])
        if code:
            raise ValueError(_status_error(code).args[0])
        fields = out[0].cpu().numpy()
    names = [COMP_NAMES[c] for c in plan.component_ids]
    components: dict[str, Any] = {}
    eta_plus = np.zeros((ny, nx), dtype=complex)
    psi_plus = np.zeros_like(eta_plus)
    for k, name in enumerate(names):
        components[name + "_plus"] = fields[k]
        components[name] = np.real(fields[k])
        if name.startswith("eta"):
            eta_plus += fields[k]
        else:
            psi_plus += fields[k]
    components["eta_plus"] = eta_plus
    components["psi_plus"] = psi_plus
    components["eta"] = np.real(eta_plus)
    components["psi"] = np.real(psi_plus)
    x, y = _xy(lx, ly, nx, ny)
    audit = {
        "implementation": "gl-b200-cuda-directional-spatial",
        "order": order,
        "grid": [ny, nx],
        "domain": [ly, lx],
        "time": float(time),
        "input": "real eta1(x,y) strict-forward in x",
        "input_reconstruction_relative": err,
        "phase_convention": "exp(i*(kx*x+ky*y)-i*omega*t)",
        "stokes_correction": False,
        "engine": {"product_grid": [plan.info.ncy, plan.info.ncx], "parent_box": list(box),
                   "precision": "fp64"},
    }
    return DirectionalFieldResult(x=x, y=y, eta=components["eta"], psi=components["psi"],
                                  components=components, audit=audit)


def gauss_laguerre_rule(rank: int):
    """Native FP64 Golub--Welsch Gauss--Laguerre rule (``quadrature.py:11-31``)."""
    lib = _lib.load()
    nodes = (C.c_double * rank)()
    weights = (C.c_double * rank)()
    status = lib.gl_gauss_laguerre(int(rank), nodes, weights)
    if status != 0:
        raise ArithmeticError(_lib.last_error())
    return np.array(nodes[:]), np.array(weights[:])


def dimensionless_wavenumber_from_frequency(omega, *, depth: float, gravity: float = 9.81):
    """Native FP64 Newton solve of ``q tanh q = omega^2 h/g`` (``dispersion.py:19-42``)."""
    lib = _lib.load()
    om = np.ascontiguousarray(np.atleast_1d(np.asarray(omega, dtype=float)))
    out = np.empty_like(om)
    status = lib.gl_dispersion_solve(int(om.size), om.ctypes.data_as(C.POINTER(C.c_double)),
                                     float(depth), float(gravity),
                                     out.ctypes.data_as(C.POINTER(C.c_double)))
    if status != 0:
        msg = _lib.last_error()
        if "converge" in msg:
            raise ArithmeticError(msg)
        raise ValueError(msg)
    return out.reshape(np.shape(omega)) if np.ndim(omega) else float(out[0])
