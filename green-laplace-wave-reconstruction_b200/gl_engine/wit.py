"""Fourth-order WIT quartet sum (sector 44) on the GPU, and the reference's
binary file formats for it.

* :func:`wit_eta44` runs ``gl_wit_eta44`` (CUDA, FP64) on a mode table and
  one or more amplitude cases;
* :func:`write_dir4in` / :func:`read_dir4in` / :func:`read_dir4out` restate
  the ``DIR4IN01`` input and ``DIR4xO01`` output layouts of
  ``paper/order4/cpp/directional_eta4_openmp.cpp:518-557, 747-773`` (writer
  ``paper/order4/write_directional_eta4_cpp_input.m``), so the engine can be
  dropped in behind the reference's ``run_cpp.py wit`` flow.
"""

from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib

FIELDS = ("eta", "psi", "eta_coordinate", "psi_coordinate", "retained")


@dataclass
class WitInput:
    modes: np.ndarray        # (M, 2) int32 mode numbers (mx, my)
    amplitudes: np.ndarray   # (cases, M) complex128
    nx: int
    ny: int
    gravity: float
    depth: float
    dkx: float
    dky: float
    threshold: float


def write_dir4in(path, inp: WitInput) -> None:
    """``DIR4IN01``: magic, (M, nx, ny, cases) uint64, (g, h, dkx, dky, thr)
    float64, M (mx, my) int32 pairs, then per case M (re, im) float64 pairs."""
    modes = np.ascontiguousarray(inp.modes, dtype="<i4").reshape(-1, 2)
    amps = np.ascontiguousarray(inp.amplitudes, dtype=np.complex128).reshape(-1, modes.shape[0])
    with open(path, "wb") as f:
        f.write(b"DIR4IN01")
        f.write(struct.pack("<4Q", modes.shape[0], inp.nx, inp.ny, amps.shape[0]))
        f.write(struct.pack("<5d", inp.gravity, inp.depth, inp.dkx, inp.dky, inp.threshold))
        f.write(modes.tobytes())
        f.write(np.ascontiguousarray(amps).view("<f8").tobytes())


def read_dir4in(path) -> WitInput:
    raw = Path(path).read_bytes()
    if raw[:8] != b"DIR4IN01":
        raise ValueError("directional input magic mismatch")
    m, nx, ny, cases = struct.unpack_from("<4Q", raw, 8)
    g, h, dkx, dky, thr = struct.unpack_from("<5d", raw, 40)
    off = 80
    modes = np.frombuffer(raw, dtype="<i4", count=2 * m, offset=off).reshape(m, 2).copy()
    off += 8 * m
    vals = np.frombuffer(raw, dtype="<f8", count=2 * m * cases, offset=off)
    amps = (vals[0::2] + 1j * vals[1::2]).reshape(cases, m)
    return WitInput(modes=modes, amplitudes=amps, nx=int(nx), ny=int(ny), gravity=g, depth=h,
                    dkx=dkx, dky=dky, threshold=thr)


@dataclass
class WitOutput:
    fields: dict             # name -> (cases, ny, nx) complex128
    stats: dict


def read_dir4out(path) -> WitOutput:
    """``DIR4xO01``: magic, 8 uint64 counters, 4 float64 diagnostics, then the
    five complex fields (eta, psi, etaCoordinate, psiCoordinate, retained),
    each [case][iy][ix]."""
    raw = Path(path).read_bytes()
    if raw[:3] != b"DIR" or raw[5:8] != b"O01":
        raise ValueError("directional output magic mismatch")
    nx, ny, cases, total, kept, near, szo, szi = struct.unpack_from("<8Q", raw, 8)
    seconds, max_res, min_det, max_src = struct.unpack_from("<4d", raw, 72)
    plane = cases * nx * ny
    vals = np.frombuffer(raw, dtype="<f8", count=10 * plane, offset=104)
    fields = {}
    for k, name in enumerate(FIELDS):
        part = vals[2 * k * plane:2 * (k + 1) * plane]
        fields[name] = (part[0::2] + 1j * part[1::2]).reshape(cases, ny, nx)
    stats = {"candidates": total, "kept": kept, "near": near, "strict_zero_output": szo,
             "strict_zero_intermediate": szi, "seconds": seconds, "max_residual": max_res,
             "min_detuning": min_det, "max_strict_zero_source": max_src}
    return WitOutput(fields=fields, stats=stats)


def write_dir4out(path, sector: int, out: WitOutput, nx: int, ny: int) -> None:
    """``DIR4xO01`` writer, the layout :func:`read_dir4out` reads."""
    st = out.stats
    cases = next(iter(out.fields.values())).shape[0]
    with open(path, "wb") as f:
        f.write({40: b"DIR40O01", 42: b"DIR42O01", 44: b"DIR44O01"}[int(sector)])
        f.write(struct.pack("<8Q", nx, ny, cases, int(st["candidates"]), int(st["kept"]),
                            int(st["near"]), int(st["strict_zero_output"]),
                            int(st["strict_zero_intermediate"])))
        f.write(struct.pack("<4d", float(st.get("seconds", 0.0)), float(st["max_residual"]),
                            float(st["min_detuning"]), float(st["max_strict_zero_source"])))
        for name in FIELDS:
            f.write(np.ascontiguousarray(out.fields[name], dtype=np.complex128).view("<f8").tobytes())


def main(argv=None) -> int:
    """Command-line twin of the reference's ``wit_eta44`` executable
    (``paper/order4/cpp/directional_eta4_openmp.cpp:499-516``):
    ``INPUT OUTPUT [--sector 40|42|44]`` (default sector 40), DIR4IN01 in,
    DIR4xO01 out, the engine's GPU direct sum in between."""
    import sys
    import time

    argv = list(sys.argv if argv is None else argv)
    if len(argv) < 3:
        print("input output [--sector 40|42|44]", file=sys.stderr)
        return 2
    sector = 40
    k = 3
    while k < len(argv):
        if argv[k] == "--sector" and k + 1 < len(argv):
            sector = int(argv[k + 1])
            k += 1
        elif argv[k].startswith("--sector="):
            sector = int(argv[k][9:])
        k += 1
    try:
        if sector not in (40, 42, 44):
            raise ValueError("sector must be 40, 42, or 44")
        inp = read_dir4in(argv[1])
        t0 = time.perf_counter()
        out = wit_sector(inp, sector)
        out.stats["seconds"] = time.perf_counter() - t0
        write_dir4out(argv[2], sector, out, inp.nx, inp.ny)
    except Exception as exc:  # the reference's error line and exit code
        print(f"DIRECTIONAL_CPP_ERROR {exc}", file=sys.stderr)
        return 1
    st = out.stats
    print(f"DIRECTIONAL_CPP_DONE sector={sector} cases={inp.amplitudes.shape[0]} "
          f"total={st['candidates']} kept={st['kept']} near={st['near']} "
          f"seconds={st['seconds']} residual={st['max_residual']}", file=sys.stderr)
    return 0


def candidates(sector: int, n_modes: int) -> int:
    """Size of a sector's quartet index space (``gl_wit_candidates``)."""
    return int(_lib.load().gl_wit_candidates(int(sector), int(n_modes)))


def wit_sector(inp: WitInput, sector: int = 44, *, device=None, as_numpy: bool = True,
               q_range: tuple[int, int] | None = None) -> WitOutput:
    """WIT fourth-order fields of one sector (44, 40 or 42) for every amplitude case.

    ``q_range`` = (begin, end) restricts the sum to those candidate indices
    (a rank's share, ``gl_wit_sector_range``); the statistics then count that
    share only."""
    lib = _lib.load()
    dev = torch.device(device if device is not None else "cuda")
    modes = np.ascontiguousarray(inp.modes, dtype=np.int32).reshape(-1, 2)
    amps = np.ascontiguousarray(inp.amplitudes, dtype=np.complex128).reshape(-1, modes.shape[0])
    m, cases = modes.shape[0], amps.shape[0]
    total = candidates(sector, m)
    q0, q1 = (0, total) if q_range is None else (int(q_range[0]), int(q_range[1]))
    with torch.cuda.device(dev):
        d_modes = torch.from_numpy(modes).to(dev)
        d_amp = torch.from_numpy(amps).to(dev)
        out = torch.empty((5, cases, inp.ny, inp.nx), dtype=torch.complex128, device=dev)
        work = torch.empty(int(lib.gl_wit_workspace_size(m)) + 256, dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.gl_wit_sector_range(int(sector), m, C.c_void_p(d_modes.data_ptr()), cases,
                                           C.c_void_p(d_amp.data_ptr()), inp.nx, inp.ny,
                                           inp.gravity, inp.depth, inp.dkx, inp.dky, inp.threshold,
                                           q0, q1, C.c_void_p(out.data_ptr()),
                                           C.c_void_p(work.data_ptr()), work.numel(),
                                           C.c_void_p(stream)))
        torch.cuda.current_stream(dev).synchronize()
        st = _lib.WitStats()
        _lib.check(lib.gl_wit_read_sector_stats(int(sector), C.c_void_p(work.data_ptr()), m,
                                                C.byref(st)))
    stats = {name: getattr(st, name) for name, _ in _lib.WitStats._fields_}
    stats["candidates"] = q1 - q0
    data = out.cpu().numpy() if as_numpy else out
    return WitOutput(fields={name: data[k] for k, name in enumerate(FIELDS)}, stats=stats)


def wit_eta44(inp: WitInput, *, device=None, as_numpy: bool = True) -> WitOutput:
    """Sector-44 WIT fields of every amplitude case on one GPU."""
    return wit_sector(inp, 44, device=device, as_numpy=as_numpy)
