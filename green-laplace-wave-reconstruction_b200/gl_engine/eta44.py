"""Fourth-order GL eta44 (no Stokes corrections) on the GPU, and the
reference's binary formats for it.

* :func:`eta44` runs a ``gl_eta44_plan_create`` plan through ``gl_execute``;
* :func:`read_glrti` / :func:`write_glrti` / :func:`read_gle44` /
  :func:`write_gle44` restate the ``GLRTI001`` input and ``GLE44O01`` output
  layouts of ``paper/order4/cpp/gl_eta44_fftw.cpp:648-691, 753-764`` (writer
  ``paper/order4/export_cpp_gl_runtime_input.m``).  Those files store arrays
  x-major (flat index ix*n + iy); this module returns numpy ``[iy, ix]``.
"""

from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .api import Plan, _engine_call, _status_error


@dataclass
class GlInput:
    n: int
    dk: float
    depth: float
    peak_depth: float
    rules: dict            # rank -> (nodes, weights)
    spectrum: np.ndarray   # [iy, ix] complex128, N^2-scaled


def write_glrti(path, inp: GlInput) -> None:
    with open(path, "wb") as f:
        f.write(b"GLRTI001")
        f.write(struct.pack("<Q3d", inp.n, inp.dk, inp.depth, inp.peak_depth))
        f.write(struct.pack("<Q", len(inp.rules)))
        for rank in sorted(inp.rules):
            nodes, weights = inp.rules[rank]
            f.write(struct.pack("<Q", rank))
            f.write(np.asarray(nodes, dtype="<f8").tobytes())
            f.write(np.asarray(weights, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(inp.spectrum.T).astype(np.complex128).view("<f8").tobytes())


def read_glrti(path) -> GlInput:
    raw = Path(path).read_bytes()
    if raw[:8] != b"GLRTI001":
        raise ValueError("magic")
    n, dk, depth, peak = struct.unpack_from("<Q3d", raw, 8)
    (nr,) = struct.unpack_from("<Q", raw, 40)
    off = 48
    rules = {}
    for _ in range(nr):
        (j,) = struct.unpack_from("<Q", raw, off)
        off += 8
        nodes = np.frombuffer(raw, "<f8", j, off).copy()
        off += 8 * j
        weights = np.frombuffer(raw, "<f8", j, off).copy()
        off += 8 * j
        rules[int(j)] = (nodes, weights)
    vals = np.frombuffer(raw, "<f8", 2 * n * n, off)
    spec = (vals[0::2] + 1j * vals[1::2]).reshape(n, n).T.copy()
    return GlInput(n=int(n), dk=dk, depth=depth, peak_depth=peak, rules=rules, spectrum=spec)


def write_gle44(path, n: int, rank: int, field: np.ndarray, threads: int = 1,
                elapsed: float = 0.0) -> None:
    """``GLE44O01``: dimensionless analytic eta44 field, x-major."""
    with open(path, "wb") as f:
        f.write(b"GLE44O01")
        f.write(struct.pack("<3Qd", n, rank, threads, elapsed))
        f.write(np.ascontiguousarray(np.asarray(field).T).astype(np.complex128).view("<f8").tobytes())


def read_gle44(path):
    raw = Path(path).read_bytes()
    if raw[:8] != b"GLE44O01":
        raise ValueError("magic")
    n, rank, threads, elapsed = struct.unpack_from("<3Qd", raw, 8)
    vals = np.frombuffer(raw, "<f8", 2 * n * n, 40)
    field = (vals[0::2] + 1j * vals[1::2]).reshape(n, n).T.copy()
    return {"n": int(n), "rank": int(rank), "threads": int(threads), "elapsed": elapsed,
            "field": field}


def spectrum_from_modes(modes, amplitudes, n: int, depth: float) -> np.ndarray:
    """s = n^2 c / h at (my, mx) (``paper/order4/prepare_order4_inputs.m:12-16``)."""
    s = np.zeros((n, n), dtype=complex)
    for (mx, my), c in zip(np.asarray(modes), np.asarray(amplitudes)):
        s[int(my) % n, int(mx) % n] = n * n * c / depth
    return s


def _box(spectrum: np.ndarray):
    n = spectrum.shape[0]
    mag = np.abs(spectrum)
    thr = 1e-13 * max(1.0, float(mag.max()))
    rows = np.flatnonzero((mag > 0).any(axis=1))
    cols = np.flatnonzero((mag > 0).any(axis=0))
    my = np.where(rows < n // 2, rows, rows - n)
    mx = np.where(cols < n // 2, cols, cols - n)
    if not np.any(mag > thr):
        raise ValueError("empty analytic support")
    return int(mx.min()), int(my.min()), int(mx.max() - mx.min() + 1), int(my.max() - my.min() + 1)


class Eta44Plan(Plan):
    def __init__(self, desc: _lib.Eta44Desc, device: torch.device, keep=None):
        self.lib = _lib.load()
        self.device = device
        self.desc = desc
        self._keep = keep
        with torch.cuda.device(device):
            handle = C.c_void_p()
            _engine_call(self.lib.gl_eta44_plan_create(C.byref(handle), C.byref(desc)))
            self.handle = handle
            info = _lib.PlanInfo()
            _engine_call(self.lib.gl_plan_get_info(handle, C.byref(info)))
            self.info = info
            size = C.c_size_t()
            _engine_call(self.lib.gl_workspace_size(handle, C.byref(size)))
            self.workspace_bytes = int(size.value)
            self._workspace = None


def eta44(spectra, *, dk: float, depth: float, peak_depth: float, rank: int, nodes=None,
          weights=None, device=None, output: str = "complex", psi44: bool = False,
          gravity: float = 1.0):
    """Physical analytic eta44 fields (depth x the GLE44O01 field) of one or
    more N^2-scaled analytic spectra ``[..., iy, ix]`` sharing one grid.

    With ``psi44=True`` returns ``(eta44, psi44)``; psi44 is the surface
    potential of ``src/gl_pure_sum_order4.m`` scaled by depth sqrt(g depth)."""
    spectra = np.asarray(spectra, dtype=np.complex128)
    single = spectra.ndim == 2
    if single:
        spectra = spectra[None]
    units, n, _ = spectra.shape
    box = _box(np.abs(spectra).max(axis=0))
    dev = torch.device(device if device is not None else "cuda")
    keep = None
    nd = wd = None
    if nodes is not None:
        keep = (np.ascontiguousarray(nodes, dtype=float), np.ascontiguousarray(weights, dtype=float))
        nd = keep[0].ctypes.data_as(C.POINTER(C.c_double))
        wd = keep[1].ctypes.data_as(C.POINTER(C.c_double))
    out_mode = _lib.OUT_REAL if output == "real" else _lib.OUT_COMPLEX
    comps = _lib.COMP_ETA44 | (_lib.COMP_PSI44 if psi44 else 0)
    desc = _lib.Eta44Desc(n=n, dk=dk, depth=depth, peak_depth=peak_depth, rank=rank, nodes=nd,
                          weights=wd, box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3],
                          max_units=1, output=out_mode, components=comps, gravity=gravity)
    plan = Eta44Plan(desc, dev, keep)
    ncomp = 2 if psi44 else 1
    with torch.cuda.device(dev):
        spec = torch.from_numpy(np.ascontiguousarray(spectra)).to(dev)
        dtype = torch.float64 if out_mode == _lib.OUT_REAL else torch.complex128
        out = torch.empty((units, ncomp, n, n), dtype=dtype, device=dev)
        status = torch.zeros(units, dtype=torch.int32, device=dev)
        plan.execute(units, torch.view_as_real(spec), _lib.SPECTRA_FULL, out, status,
                     torch.cuda.current_stream(dev).cuda_stream)
        st = status.cpu().numpy()
        if np.any(st != 0):
            raise _status_error(int(st[st != 0][0]))
        res = out.cpu().numpy()
    if single:
        res = res[0]
        return (res[0], res[1]) if psi44 else res[0]
    return (res[:, 0], res[:, 1]) if psi44 else res[:, 0]


def eta44_part(spectrum, *, dk: float, depth: float, peak_depth: float, rank: int, outer: int,
               part: int = -2, nodes=None, weights=None, device=None) -> np.ndarray:
    """Physical analytic eta44 field of one part of the reference's split mode
    (``paper/order4/cpp/gl_eta44_fftw.cpp:639-749``): outer GL node ``outer``
    alone; ``part`` -2 every forcing partition, -1 the base partitions 22,
    211 and 1111, t >= 0 partition 31 with third-level node t alone.  The
    part's spectrum gets its own final roundoff floor, as each split process
    of the reference does; summing the parts' fields is what
    ``merge_eta44_outer`` does (``merge_main``)."""
    spectrum = np.asarray(spectrum, dtype=np.complex128)
    n = spectrum.shape[0]
    box = _box(np.abs(spectrum))
    dev = torch.device(device if device is not None else "cuda")
    keep = None
    nd = wd = None
    if nodes is not None:
        keep = (np.ascontiguousarray(nodes, dtype=float), np.ascontiguousarray(weights, dtype=float))
        nd = keep[0].ctypes.data_as(C.POINTER(C.c_double))
        wd = keep[1].ctypes.data_as(C.POINTER(C.c_double))
    desc = _lib.Eta44Desc(n=n, dk=dk, depth=depth, peak_depth=peak_depth, rank=rank, nodes=nd,
                          weights=wd, box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3],
                          max_units=1, output=_lib.OUT_COMPLEX, components=_lib.COMP_ETA44,
                          gravity=1.0)
    plan = Eta44Plan(desc, dev, keep)
    lib = plan.lib
    b4 = (4 * (box[3] - 1) + 1, 4 * (box[2] - 1) + 1)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        spec = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(spectrum[None])).to(dev))
        partial = torch.zeros((1, 1) + b4, dtype=torch.complex128, device=dev)
        out = torch.empty((1, 1, n, n), dtype=torch.complex128, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _engine_call(lib.gl_eta44_execute_part(
            plan.handle, 1, C.c_void_p(spec.data_ptr()), _lib.SPECTRA_FULL, int(outer), int(part),
            C.c_void_p(partial.data_ptr()), C.c_void_p(plan._ws_ptr()),
            C.c_size_t(plan.workspace_bytes), C.c_void_p(status.data_ptr()), C.c_void_p(stream)))
        _engine_call(lib.gl_eta44_finalize(
            plan.handle, 1, C.c_void_p(partial.data_ptr()), C.c_void_p(out.data_ptr()),
            C.c_void_p(plan._ws_ptr()), C.c_size_t(plan.workspace_bytes), C.c_void_p(stream)))
        st = int(status.item())
        if st != 0:
            raise _status_error(st)
        return out[0, 0].cpu().numpy()


def gl_pure_sum_order4(s, qx, qy, qp: float, rank: int = 4, *, device=None):
    """``[eta44, psi44, audit] = gl_pure_sum_order4(s, qx, qy, qp, rank)``
    (``src/gl_pure_sum_order4.m:1-15``): dimensionless analytic eta44/h and
    psi44/(h sqrt(gh)) of ``s = fft2(eta11_plus/h)`` on the grid ``qx = kx h``,
    ``qy = ky h`` (square, power-of-two, equal spacing in x and y), peak
    ``qp = kp h``, one GL rank for all three nested levels."""
    s = np.asarray(s, dtype=np.complex128)
    qx = np.asarray(qx, dtype=float)
    qy = np.asarray(qy, dtype=float)
    if rank not in (4, 6, 8, 10, 12):
        raise ValueError("Unsupported no-Stokes order-four Green--Laplace rank.")
    if not (s.shape == qx.shape == qy.shape) or s.ndim != 2 or s.shape[0] != s.shape[1]:
        raise ValueError("Spectrum, qx, and qy must have identical square sizes.")
    dq = float(qx[0, 1] - qx[0, 0])
    if not (dq > 0) or abs(float(qy[1, 0] - qy[0, 0]) - dq) > 1e-12 * dq:
        raise ValueError("qx and qy must be the fft2 wavenumber grids of one square lattice")
    eta, psi = eta44(s, dk=dq, depth=1.0, peak_depth=float(qp), rank=rank, device=device,
                     psi44=True, gravity=1.0)
    audit = {"implementation": "no-stokes-green-laplace-order4", "quadrature_rank": rank,
             "nested_rank_tuple": (rank, rank, rank), "order4_stokes_correction_used": False,
             "release_status": "experimental no-Stokes migration; not a total-field API extension"}
    return eta, psi, audit


def main(argv=None) -> int:
    """Command-line twin of the reference's ``gl_eta44`` executable
    (``paper/order4/cpp/gl_eta44_fftw.cpp:639-764``):
    ``INPUT OUTPUT RANK THREADS [OUTER4_INDEX [PART_INDEX]]``, GLRTI001 in
    (the rule of RANK taken from the file), GLE44O01 out (the dimensionless
    field).  With OUTER4_INDEX (and PART_INDEX) it computes that part of the
    split mode (``eta44_part``), so the reference's split launcher
    (``paper/order4/run_gl_split.sh``) and merger can drive it."""
    import sys
    import time

    argv = list(sys.argv if argv is None else argv)
    try:
        if len(argv) not in (5, 6, 7):
            raise ValueError("usage INPUT OUTPUT RANK THREADS [OUTER4_INDEX [PART_INDEX]]")
        rank, threads = int(argv[3]), int(argv[4])
        requested = int(argv[5]) if len(argv) >= 6 else -1
        part = int(argv[6]) if len(argv) == 7 else -2
        if requested >= rank:
            raise ValueError("outer index")
        if part >= rank or part < -2:
            raise ValueError("part index")
        if len(argv) == 7 and requested < 0:
            raise ValueError("split mode requires one outer4 index")
        inp = read_glrti(argv[1])
        if rank not in inp.rules:
            raise ValueError("rank")
        nodes, weights = inp.rules[rank]
        t0 = time.perf_counter()
        if requested >= 0:
            field = eta44_part(inp.spectrum, dk=inp.dk, depth=inp.depth,
                               peak_depth=inp.peak_depth, rank=rank, outer=requested, part=part,
                               nodes=nodes, weights=weights) / inp.depth
        else:
            field = eta44(inp.spectrum, dk=inp.dk, depth=inp.depth, peak_depth=inp.peak_depth,
                          rank=rank, nodes=nodes, weights=weights) / inp.depth
        elapsed = time.perf_counter() - t0
        write_gle44(argv[2], inp.n, rank, field, threads=threads, elapsed=elapsed)
    except Exception as exc:  # the reference's error line and exit code
        print(f"CPP_GL_ETA44_ERROR {exc}", file=sys.stderr)
        return 1
    print(f"CPP_GL_ETA44_DONE n={inp.n} rank={rank} threads={threads} outer={requested} "
          f"part={part} elapsed={elapsed}", file=sys.stderr)
    return 0


def merge_main(argv=None) -> int:
    """Command-line twin of the reference's ``merge_eta44_outer``
    (``paper/order4/cpp/merge_eta44_outer.cpp:12``): ``OUTPUT INPUT1 INPUT2
    ...``; sums the GLE44O01 fields of the split parts (same n and rank),
    writes one GLE44O01 whose thread slot holds the part count and whose time
    is the slowest part's."""
    import sys

    argv = list(sys.argv if argv is None else argv)
    try:
        if len(argv) < 4:
            raise ValueError("usage OUTPUT INPUT1 INPUT2 ...")
        total, n, rank, wall = None, 0, 0, 0.0
        for path in argv[2:]:
            part = read_gle44(path)
            if total is None:
                n, rank, total = part["n"], part["rank"], np.zeros((part["n"], part["n"]), complex)
            elif part["n"] != n or part["rank"] != rank:
                raise ValueError("incompatible partial outputs")
            wall = max(wall, part["elapsed"])
            total = total + part["field"]
        write_gle44(argv[1], n, rank, total, threads=len(argv) - 2, elapsed=wall)
    except Exception as exc:
        print(f"CPP_GL_ETA44_MERGE_ERROR {exc}", file=sys.stderr)
        return 1
    print(f"CPP_GL_ETA44_MERGE rank={rank} partials={len(argv) - 2} max_node_seconds={wall}",
          file=sys.stderr)
    return 0
