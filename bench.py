#!/usr/bin/env python
"""Throughput of the order-3 GL graph: eta33 + psi33 fields/s at 1024^2.

Workload (one "unit" = one eta33+psi33 pair from one analytic spectrum):
order-3 positive pure-sum GL4/GL4, Nx=Ny=1024, Lx=Ly=1024 m, h=30 m, 4096
JONSWAP modes (Hs=3 m, Tp=10 s, gamma 3.3, cos^20 spreading, seed 0).  A step
evaluates U time snapshots of that sea state on each GPU (units are sharded
across ranks: no collective on the data path).

Arms:
* default: the CUDA engine.  ``value`` times gl_execute on spectra already in
  HBM (CUDA events per step, L2 flushed between steps outside the events);
  ``e2e`` times the public streaming API (``SurfaceStream``) with host inputs
  and a device->host read of the real fields each step; each step's copy out
  overlaps the next step's evaluation.
* ``--impl reference``: the reference algorithm on the host CPU (the FP64
  NumPy oracle, one process per core), rank 0 only.

Prints one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "green-laplace-wave-reconstruction_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "GL4 eta33+psi33 1024² fields/s, FP32 vs FP64 on 1 B200 @≤1e-6 rel err; %HBM"
UNIT = "fields/s"
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20


def workload_config(units: int, world: int, product_grid=None) -> dict:
    cfg = {
        "workload": "order-3 eta33+psi33 GL4/GL4, 1024^2 grid, Lx=Ly=1024 m, h=30 m, 4096 JONSWAP "
                    "modes (Hs=3 m, Tp=10 s, seed 0); each step = U time snapshots per GPU",
        "units_per_step_per_gpu": units,
        "grid": [1024, 1024],
        "precision": "fp64 (all GL nodes)",
        "l2": "flushed between timed steps (256 MiB write outside the events)",
        "parallelism": f"units sharded over {world} rank(s), no data-path collective",
    }
    if product_grid is not None:
        cfg["product_grid"] = product_grid
    return cfg


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi takes a moment to start: wait for its first sample so
        # that the timed region is covered
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < 5.0:
            try:
                if Path(self.path).stat().st_size > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU leg (oracle) helpers
# ---------------------------------------------------------------------------


def _oracle_inputs(t: float):
    from gl_engine import seastate
    from oracle import gl_oracle as O

    st = seastate.config2(0)
    kxg, kyg = O.fft_wavenumber_grid(st.lx, st.ly, st.nx, st.ny)
    oc = O.spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], st.depth, st.lx, st.ly,
                        st.nx, st.ny, t)
    return st, s, st.depth * kxg, st.depth * kyg


def _oracle_part(args):
    """One worker task: the listed outer GL nodes of one unit (single thread)."""
    t, subset = args
    from oracle import gl_oracle as O

    _, s, qx, qy = _oracle_inputs(t)
    t0 = time.perf_counter()
    O.order3(s, qx, qy, outer_subset=set(subset))
    return time.perf_counter() - t0


def cpu_baseline_sample() -> tuple[dict, object]:
    """One full unit (t=0) by the FP64 oracle on one host core."""
    from oracle import gl_oracle as O

    st, s, qx, qy = _oracle_inputs(0.0)
    t0 = time.perf_counter()
    e33, p33, _ = O.order3(s, qx, qy)
    dt = time.perf_counter() - t0
    pscale = st.depth * math.sqrt(st.gravity * st.depth)
    return ({"value": 1.0 / dt, "unit": UNIT, "cores": 1, "kind": "port",
             "sample": f"1 unit (t=0 s) of the workload, full GL4/GL4 graph, {dt:.2f} s "
                       "single-threaded FP64 NumPy oracle"},
            (st.depth * e33, pscale * p33))


def _oracle_perturbed(kind: str):
    """The workload's unit by the oracle under one roundoff-level change:
    'axes' (every 2-D FFT in the other axis order) or 'floor+' / 'floor-'
    (the roundoff floor's threshold moved by one ulp of the peak)."""
    import numpy.fft as F

    from oracle import gl_oracle as O

    st, s, qx, qy = _oracle_inputs(0.0)
    f2, i2, floor0 = F.fft2, F.ifft2, O.zero_below_roundoff_floor
    ulp = 1.0 / (16.0 * math.log2(st.nx * st.ny))
    factor = {"floor+": 1.0 + ulp, "floor-": 1.0 - ulp}.get(kind, 1.0)

    def floor(spectrum, support):
        import numpy as np

        out = spectrum.copy()
        mags = np.abs(out[support])
        if mags.size == 0 or float(np.max(mags)) == 0.0:
            return out
        thr = 16.0 * O.EPS * max(1.0, np.log2(out.size)) * factor * float(np.max(mags))
        out[support & (np.abs(out) < thr)] = 0.0
        return out

    try:
        if kind == "axes":
            F.fft2 = lambda a: F.fft(F.fft(a, axis=0), axis=1)
            F.ifft2 = lambda a: F.ifft(F.ifft(a, axis=0), axis=1)
        else:
            O.zero_below_roundoff_floor = floor
        e33, p33, _ = O.order3(s, qx, qy)
    finally:
        F.fft2, F.ifft2, O.zero_below_roundoff_floor = f2, i2, floor0
    pscale = st.depth * math.sqrt(st.gravity * st.depth)
    return st.depth * e33, pscale * p33


def oracle_spread_samples():
    """The three perturbed oracle runs of the workload's unit, side by side in
    spawned processes: their distances to the plain oracle are the oracle's
    own roundoff spread on this workload."""
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(3) as pool:
        return pool.map(_oracle_perturbed, ["axes", "floor+", "floor-"])


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    workers = max(1, min(cores, 16))
    ctx = mp.get_context("spawn")
    # one step = one outer GL node (1/4 of the graph) of `workers` distinct units
    tasks = [(0.5 * k, [k % 4]) for k in range(workers)]
    with ctx.Pool(workers) as pool:
        for _ in range(args.warmup):
            pool.map(_oracle_part, tasks)
        steps = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            pool.map(_oracle_part, tasks)
            steps.append(time.perf_counter() - t0)
    total = sum(steps)
    fields = args.steps * workers * 0.25
    value = fields / total
    package = _reference_package_unit()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded JONSWAP sea state)",
        "config": workload_config(workers, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"each step: outer GL node k%4 of {workers} units (1/4 of each "
                                   "unit's graph) in parallel processes, FP64 NumPy oracle"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if package is not None:
        line["reference_package_check"] = package
    print(json.dumps(line), flush=True)


def _reference_package_unit():
    """One full unit through the reference's own Python package when it is
    installed in baseline/_ref (its ``green_laplace_order3``; the deposit is
    the oracle's restatement of the MATLAB two-stage entry, which the package
    lacks): seconds per unit next to the port's, and the two fields' distance.
    The timed arm above runs the port because the package's function has no
    per-node split to bound a step; this check shows the two run the same
    arithmetic at the same speed."""
    ref_dir = ROOT / "baseline" / "_ref"
    if not (ref_dir / "green_laplace" / "_order3.py").exists():
        return None
    import importlib

    from oracle import gl_oracle as O

    sys.path.insert(0, str(ref_dir))
    try:
        ref_order3 = importlib.import_module("green_laplace._order3")
    finally:
        sys.path.remove(str(ref_dir))
    _, s, qx, qy = _oracle_inputs(0.0)
    t0 = time.perf_counter()
    e_pkg, p_pkg, _ = ref_order3.green_laplace_order3(s, qx, qy)
    pkg_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    e_port, p_port, _ = O.order3(s, qx, qy)
    port_s = time.perf_counter() - t0
    import numpy as np

    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    return {"installed_at": "baseline/_ref/green_laplace (the reference's src tree; its hatchling "
                            "build backend is not in the offline wheelhouse)",
            "package_seconds_per_unit": pkg_s, "port_seconds_per_unit": port_s,
            "eta33_rel_l2_package_vs_port": rel(e_port, e_pkg),
            "psi33_rel_l2_package_vs_port": rel(p_port, p_pkg)}


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------


# ---------------------------------------------------------------------------
# the plain single-field GPU path (comparison leg)
# ---------------------------------------------------------------------------


def plain_gpu_order3(s, qx, qy, *, complex_dtype, floor_eps, inner_rank=4, outer_rank=4):
    """The order-3 graph of ``_order3.py:18-148`` written as plain cuFFT calls
    (torch.fft) on the full reference grid, one field at a time: no fusion, no
    compact grid, no batching.  This is the "plain single-field GPU path" the
    engine is compared with, in FP64 (complex128) or FP32 (complex64, with
    the roundoff floor scaled to the FP32 epsilon).  Returns (eta33/h,
    psi33/(h sqrt(gh))) as complex fields."""
    import numpy as np
    import torch

    from gl_engine import api

    rdt = torch.float64 if complex_dtype == torch.complex128 else torch.float32
    qx, qy = qx.to(rdt), qy.to(rdt)
    s = s.to(complex_dtype)
    tiny = torch.finfo(rdt).tiny
    q = torch.hypot(qx, qy)
    a_ = q * torch.tanh(q)
    nu = torch.sqrt(a_)
    sqa = torch.sqrt(a_)
    snu = nu.clamp_min(tiny)
    q2 = q * q
    mag = s.abs()
    support = mag > 1e-13 * max(1.0, float(mag.max()))
    hat = torch.fft.fft2(support.to(complex_dtype))
    s2 = torch.fft.ifft2(hat * hat).real > 0.5
    s3 = torch.fft.ifft2(hat * hat * hat).real > 0.5
    nu_min = float(nu[support].min())
    shift2 = 0.5 * (nu_min + float(sqa[s2].max()) / 2.0)
    shift3 = 0.5 * (nu_min + float(sqa[s3].max()) / 3.0)
    amp2 = torch.where(support, mag * mag, torch.zeros_like(mag))
    qp = float(q.flatten()[int(torch.argmax(amp2.flatten()))])
    pn = np.sqrt(qp * np.tanh(qp))
    lam2 = 2.0 * pn - np.sqrt(2.0 * qp * np.tanh(2.0 * qp))
    lam3 = 3.0 * pn - np.sqrt(3.0 * qp * np.tanh(3.0 * qp))
    fl = 16.0 * floor_eps * max(1.0, np.log2(s.numel()))

    def sup(h, m):
        h = torch.where(m, h, torch.zeros_like(h))
        peak = float(h.abs().max())
        return h if peak == 0.0 else torch.where(m & (h.abs() < fl * peak), torch.zeros_like(h), h)

    def shr(t):
        return torch.where(sqa > 0, torch.sinh(sqa * t) / sqa.clamp_min(tiny), torch.full_like(sqa, t))

    ifft, fft = torch.fft.ifft2, torch.fft.fft2
    inodes, iweights = api.gauss_laguerre_rule(inner_rank)
    onodes, oweights = api.gauss_laguerre_rule(outer_rank)
    eta_hat = torch.zeros_like(s)
    psi_hat = torch.zeros_like(s)
    for x, w in zip(onodes, oweights):
        tau = x / lam3
        d = s * torch.exp(-tau * (nu - shift3))
        f = {"eta": ifft(d), "etax": ifft(1j * qx * d), "etay": ifft(1j * qy * d),
             "phix": ifft(qx / snu * d), "phiy": ifft(qy / snu * d), "phiz": ifft(-1j * nu * d),
             "phixz": ifft(nu * qx * d), "phiyz": ifft(nu * qy * d),
             "phizz": ifft(-1j * q2 / snu * d), "phizzz": ifft(-1j * q2 * nu * d),
             "phitz": ifft(-a_ * d), "phitzz": ifft(-q2 * d)}
        e_h = torch.zeros_like(s)
        et_h = torch.zeros_like(s)
        p_h = torch.zeros_like(s)
        pt_h = torch.zeros_like(s)
        for xi, wi in zip(inodes, iweights):
            t2 = xi / lam2
            d2 = d * torch.exp(-t2 * (nu - shift2))
            v, v1, v2, v3 = ifft(d2), ifft(d2 * nu), ifft(d2 * nu * nu), ifft(d2 * nu ** 3)
            hx, hy, jx, jy = ifft(d2 * qx / snu), ifft(d2 * qy / snu), ifft(d2 * qx), ifft(d2 * qy)
            rad, qq, njx, njy = ifft(d2 * q2 / snu), ifft(d2 * q2), ifft(d2 * nu * qx), ifft(d2 * nu * qy)
            srcs = (2 * v * v2 + v1 * v1 - hx * hx - hy * hy,
                    2 * v * rad + 2 * (hx * jx + hy * jy),
                    2 * v * v3 + 4 * v1 * v2 - 2 * hx * jx - 2 * hy * jy,
                    2 * (v1 * rad + v * qq) + 2 * (jx * jx + hx * njx + jy * jy + hy * njy))
            sd, sk, sdt, skt = (sup(fft(x_), s2) for x_ in srcs)
            sh, ch = shr(t2), torch.cosh(sqa * t2)
            c = wi * np.exp(xi) / lam2 * np.exp(-2.0 * shift2 * t2) / 4.0
            e_h = e_h + c * (-a_ * sh * sd + ch * sk)
            et_h = et_h - 1j * c * (-a_ * sh * sdt + ch * skt)
            p_h = p_h + 1j * c * (ch * sd - sh * sk)
            pt_h = pt_h + c * (ch * sdt - sh * skt)
        et_h = sup(et_h, s2)
        p = {"eta": ifft(e_h), "etax": ifft(1j * qx * e_h), "etay": ifft(1j * qy * e_h),
             "phix": ifft(1j * qx * p_h), "phiy": ifft(1j * qy * p_h), "phiz": ifft(a_ * p_h),
             "phizz": ifft(q2 * p_h), "phitz": ifft(a_ * pt_h), "eta_t": ifft(et_h)}
        fe = f["eta"]
        k_pair = (f["phix"] * p["etax"] + f["phiy"] * p["etay"] + p["phix"] * f["etax"]
                  + p["phiy"] * f["etay"] - fe * p["phizz"] - p["eta"] * f["phizz"])
        k_dir = fe * (f["phixz"] * f["etax"] + f["phiyz"] * f["etay"]) - 0.5 * fe * fe * f["phizzz"]
        d_pair = (fe * p["phitz"] + p["eta"] * f["phitz"] + f["phix"] * p["phix"]
                  + f["phiy"] * p["phiy"] + f["phiz"] * p["phiz"])
        d_dir = 0.5 * fe * fe * f["phitzz"] + fe * (f["phix"] * f["phixz"] + f["phiy"] * f["phiyz"]
                                                    + f["phiz"] * f["phizz"])
        cont = 0.5 * fe * p["phiz"] + 0.5 * p["eta"] * f["phiz"] + 0.125 * fe * fe * f["phizz"]
        cont_t = (0.5 * (f["phiz"] * p["phiz"] + fe * p["phitz"])
                  + 0.5 * (p["eta_t"] * f["phiz"] + p["eta"] * f["phitz"])
                  + 0.25 * fe * f["phiz"] * f["phizz"] + 0.125 * fe * fe * f["phitzz"])
        fk, fd, c_h, ct_h = (sup(fft(x_), s3) for x_ in (k_dir / 4 + k_pair / 2, d_dir / 4 + d_pair / 2,
                                                          cont, cont_t))
        fk_psi = sup(fk + a_ * c_h, s3)
        fd_psi = sup(fd - ct_h, s3)
        sh, ch = shr(tau), torch.cosh(sqa * tau)
        c = w * np.exp(x) / lam3 * np.exp(-3.0 * shift3 * tau)
        eta_hat = eta_hat + c * (a_ * sh * fd - 1j * ch * fk)
        psi_hat = psi_hat + c * (-1j * ch * fd_psi - sh * fk_psi)
    eta_hat = torch.where(s3, eta_hat, torch.zeros_like(eta_hat))
    psi_hat = torch.where(s3, psi_hat, torch.zeros_like(psi_hat))
    return ifft(eta_hat), ifft(psi_hat)


def plain_gpu_leg(plan, spectra, st, first, device) -> dict:
    """Time the plain single-field FP64 GPU path on one unit and measure the
    FP32 variant's error against the engine."""
    import numpy as np
    import torch

    box = plan.info.box1
    x0, y0, w, h = box[0], box[1], box[2], box[3]
    full = torch.zeros((st.ny, st.nx), dtype=torch.complex128, device=device)
    rows = (torch.arange(h, device=device) + y0) % st.ny
    cols = (torch.arange(w, device=device) + x0) % st.nx
    full[rows[:, None], cols[None, :]] = torch.view_as_complex(spectra[0].contiguous())
    kx = 2.0 * np.pi * np.fft.fftfreq(st.nx, d=st.lx / st.nx)
    ky = 2.0 * np.pi * np.fft.fftfreq(st.ny, d=st.ly / st.ny)
    kxg, kyg = np.meshgrid(kx, ky)
    qx = torch.as_tensor(st.depth * kxg, device=device)
    qy = torch.as_tensor(st.depth * kyg, device=device)
    hs = st.depth
    ps = st.depth * np.sqrt(st.gravity * st.depth)
    out = {}
    for name, cdt, feps in (("fp64", torch.complex128, 2.220446049250313e-16),
                            ("fp32", torch.complex64, float(np.finfo(np.float32).eps))):
        plain_gpu_order3(full, qx, qy, complex_dtype=cdt, floor_eps=feps)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        e, p = plain_gpu_order3(full, qx, qy, complex_dtype=cdt, floor_eps=feps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        e = (hs * e.real).double().cpu().numpy()
        p = (ps * p.real).double().cpu().numpy()
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        out[name] = {"fields_per_s": 1e3 / ms, "ms_per_field": ms,
                     "eta33_rel_l2_vs_engine": rel(e, first[0]),
                     "psi33_rel_l2_vs_engine": rel(p, first[1])}
    out["note"] = ("torch.fft (cuFFT) graph on the full 1024^2 grid, one field per call; fp32 = "
                   "complex64 FFTs and products with the floor scaled to the FP32 epsilon")
    return out


def run_engine(args, rank: int, world: int, local_rank: int) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist

    import gl_engine
    from gl_engine import _lib, api, seastate

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    U = args.units
    st = seastate.config2(0)
    coeffs = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    times = np.array([0.5 * (rank * U + u) for u in range(U)], dtype=np.float64)
    dep = api.prepare_deposit(coeffs, st.lx, st.ly, st.nx, st.ny)
    plan = api.get_plan(nx=st.nx, ny=st.ny, lx=st.lx, ly=st.ly, depth=st.depth,
                        gravity=st.gravity, order=3,
                        components=_lib.COMP_ETA33 | _lib.COMP_PSI33, eta22_rank=6,
                        allow_below=False, box=dep.box, grid=_lib.GRID_COMPACT,
                        max_units=args.group or U, output=_lib.OUT_REAL, device=device)
    if args.lanes > 1 and plan.lanes != args.lanes:
        plan.set_lanes(args.lanes)
    stream = torch.cuda.current_stream(device)
    dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device, dt)  # noqa: E731
    seg_off, seg_bin = dev(dep.seg_offsets, torch.int32), dev(dep.seg_bins, torch.int32)
    ab, om, tt = dev(dep.ab, torch.float64), dev(dep.omega, torch.float64), dev(times, torch.float64)
    w, h = dep.box[2], dep.box[3]
    spectra = torch.empty((U, h, w, 2), dtype=torch.float64, device=device)
    plan.deposit(U, seg_off, seg_bin, ab, om, tt, spectra, stream.cuda_stream)
    out = torch.empty((U, 2, st.ny, st.nx), dtype=torch.float64, device=device)
    status = torch.zeros(U, dtype=torch.int32, device=device)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)

    def step():
        plan.execute(U, spectra, _lib.SPECTRA_BOX, out, status, stream.cuda_stream)

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    if int(status.abs().sum()) != 0:
        raise RuntimeError(f"engine status {status.tolist()}")
    first = out[0].cpu().numpy().copy() if rank == 0 else None

    # ---- timed region: K steps, CUDA events per step on the launching stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.launch_count()
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = _lib.launch_count() - launches0
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    t_max = torch.tensor([t_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    total_s = float(t_max.item()) / 1e3
    value = U * args.steps * world / total_s
    clocks = clk.summary()

    # ---- per-kernel breakdown (separate profiled pass, events per launch).
    # Concurrent lanes overlap kernels, which would stretch each launch's
    # event-timed duration, so this pass runs the same units through a
    # one-lane plan of the same shape: every kernel then runs alone, as in an
    # ncu launch list.
    prof_plan = api.Plan(plan.desc, device) if plan.lanes > 1 else plan
    _lib.profile_begin()
    for _ in range(2):
        prof_plan.execute(U, spectra, _lib.SPECTRA_BOX, out, status, stream.cuda_stream)
    torch.cuda.synchronize()
    kstats = _lib.profile_end()
    del prof_plan
    kstats.sort(key=lambda r: -r["ms_total"])
    tot = sum(r["ms_total"] for r in kstats) or 1.0
    top = kstats[0]
    peak, peak_src = measured_peaks()
    achieved = top["bytes_total"] / (top["ms_total"] / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "dram_traffic.json"
    if tfile.exists():
        try:
            tdat = json.loads(tfile.read_text())
            per = tdat.get(top["name"])
            if per is not None:
                traffic = float(per["bytes_per_unit"]) * plan.desc.max_units
        except Exception:
            traffic = None
    roofline = {
        "bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak,
        "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
        "traffic": traffic,
        "algorithmic_bytes_per_launch": top["bytes_total"] / top["launches"],
        "avg_launch_ms": top["ms_total"] / top["launches"],
        "kernel_shares": [{"name": r["name"], "launches": r["launches"],
                           "share": round(r["ms_total"] / tot, 4)} for r in kstats[:8]],
    }
    # the reference's dense-transform accounting (358 transforms x 2 passes x
    # (read+write) x N^2 x 16 B per unit), for comparison only
    dense_bytes = 358 * 2 * 2 * st.nx * st.ny * 16
    accounting = {"dense_reference_bytes_per_unit": dense_bytes,
                  "dense_equivalent_gbs": dense_bytes * value / 1e9,
                  "product_grid": [plan.info.ncy, plan.info.ncx]}

    # ---- end to end through the public API, host inputs -> host fields
    e2e = None
    if not args.no_e2e:
        h2d = dep.ab.nbytes + dep.omega.nbytes + dep.seg_offsets.nbytes + dep.seg_bins.nbytes + \
            times.nbytes
        d2h = U * 2 * st.ny * st.nx * 8
        # the public streaming API: every step copies its inputs in and its
        # real fields out to pinned host memory; step i's device->host copy
        # overlaps step i+1's evaluation
        sstream = api.SurfaceStream(coeffs, st.lx, st.ly, st.nx, st.ny,
                                    components=["eta33", "psi33"], output="real", device=device,
                                    max_units=args.group or U, check=False)

        def e2e_steps(k):
            pending = None
            for _ in range(k):
                ticket = sstream.submit(times)
                if pending is not None:
                    sstream.result(pending)
                pending = ticket
            sstream.result(pending)

        e2e_steps(2)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_steps(args.steps)
        torch.cuda.synchronize()
        e2e_s = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=device)
        if world > 1:
            dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
        e2e = {"value": U * args.steps * world / float(e2e_s.item()), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}
        # the host link's own bound on this figure: a plain device->pinned-host
        # copy of one step's fields, timed on a copy stream
        host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
        cs = torch.cuda.Stream(device)
        cs.wait_stream(stream)
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(cs):
            host.copy_(out, non_blocking=True)
            l0.record(cs)
            for _ in range(4):
                host.copy_(out, non_blocking=True)
            l1.record(cs)
        torch.cuda.synchronize()
        link_gbs = 4 * d2h / (l0.elapsed_time(l1) / 1e3) / 1e9
        e2e["d2h_link_gbs"] = link_gbs
        e2e["link_bound"] = {
            "value": U * world / (d2h / (link_gbs * 1e9)), "unit": UNIT,
            "note": "fields/s if every step's device->host copy ran back to back at the measured "
                    "link rate; the streamed copies overlap the next step's evaluation, so the "
                    "end-to-end figure is bounded by the host link, not the kernels"}
        del host

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded JONSWAP + cos^2s sea state; no dataset)",
        "config": dict(workload_config(U, world, [plan.info.ncy, plan.info.ncx]),
                       lanes=f"{plan.lanes} concurrent lane(s) of {plan.desc.max_units // plan.lanes} "
                             "units per engine launch"),
        "roofline": roofline, "accounting": accounting, "clocks": clocks,
        "gpu_launches": int(launches), "e2e": e2e,
    }
    if world == 1 and not args.no_plain_gpu:
        plain = plain_gpu_leg(plan, spectra, st, first, device)
        line["plain_gpu_path"] = plain
        line["speedup_vs_plain_fp64_gpu"] = value / plain["fp64"]["fields_per_s"]
    if world == 1 and not args.no_cpu_baseline:
        base, (e_ref, p_ref) = cpu_baseline_sample()
        line["cpu_baseline"] = base
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        mrel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))  # noqa: E731
        # the oracle's own roundoff spread on this workload: the same unit with
        # the 2-D FFTs in the other axis order, and with the roundoff floor's
        # threshold moved by one ulp of the peak either way
        alts = oracle_spread_samples()
        spread = {"eta33": max(rel(e.real, e_ref.real) for e, _ in alts),
                  "psi33": max(rel(p.real, p_ref.real) for _, p in alts)}
        line["parity_vs_oracle"] = {
            name: {"rel_l2": rel(got, ref.real), "max_abs_rel": mrel(got, ref.real),
                   "oracle_roundoff_spread": spread[name]}
            for name, got, ref in (("eta33", first[0], e_ref), ("psi33", first[1], p_ref))}
        line["parity_vs_oracle"]["precision"] = {
            "fp64_nodes": "all (4 outer x 4 inner GL nodes and every transform)",
            "fp32_nodes": [],
            "why": "oracle/node_precision.py on this workload: one node in complex64 at a time "
                   "moves eta33 by 2.3e-7 (outer node 1) up to 3e32 (inner node 4 of outer node 4); "
                   "only outer node 1 stays under 1e-6 on its own (6.9 % of the transforms)"}
    print(json.dumps(line), flush=True)


def run_config3(args, rank: int, world: int, local_rank: int) -> None:
    """The uneven batch (64 sea states, grids 128..1024^2, orders 2-3, ranks
    2..8, 8 snapshots each) replayed as one captured CUDA graph, against the
    same batch launched eagerly.  Units = (sea state, snapshot) pairs."""
    import torch

    from gl_engine import _lib, batch

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    items = batch.config3_items(n_states=args.states, snapshots=8, seed0=rank * args.states)
    t_tune = time.perf_counter()
    lanes = batch.autotune_lanes(items, candidates=(1, 2, 4, 8, 12, 16), device=device)
    t_tune = time.perf_counter() - t_tune
    t_tiles = time.perf_counter()
    runner = batch.BatchRunner(items, device=device, lanes=lanes, tiles="auto")
    t_tiles = time.perf_counter() - t_tiles
    tuned = sum(1 for s in runner.staged if any(getattr(s.plan, "tuning", (0, 0, 0))))
    runner.capture()
    for _ in range(max(args.warmup, 1)):
        runner.replay()
    torch.cuda.synchronize()
    runner.check()
    stream = torch.cuda.current_stream(device)

    def timed(fn):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        for k in range(args.steps):
            ev[k][0].record(stream)
            fn()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / 1e3

    launches0 = _lib.launch_count()
    eager_s = timed(runner.run_eager)
    launches = (_lib.launch_count() - launches0) // max(args.steps, 1)
    graph_s = timed(runner.replay)
    units = runner.units
    grids = sorted({it.nx for it in items})
    # per-kernel breakdown: one profiled eager pass (events per launch)
    _lib.profile_begin()
    runner.run_eager()
    torch.cuda.synchronize()
    kstats = sorted(_lib.profile_end(), key=lambda r: -r["ms_total"])
    ktot = sum(r["ms_total"] for r in kstats) or 1.0
    # the same batch with one lane (the states one after another), and with
    # the built-in launch shapes, for reference
    serial = batch.BatchRunner(items, device=device, lanes=1, tiles="auto")
    serial.capture()
    serial.replay()
    torch.cuda.synchronize()
    serial_s = timed(serial.replay)
    del serial
    for s in runner.staged:
        s.plan.set_tuning(0, 0, 0)
    untuned = batch.BatchRunner(items, device=device, lanes=lanes)
    untuned.capture()
    untuned.replay()
    torch.cuda.synchronize()
    untuned_s = timed(untuned.replay)
    del untuned
    line = {
        "metric": "config-3 uneven batch units/s (captured graph)", "value": units * args.steps / graph_s,
        "unit": "units/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * graph_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded JONSWAP sea states)",
        "config": {"workload": f"{len(items)} sea states x 8 snapshots, grids {grids}, orders 2-3, "
                               "ranks 2-8, h U[10,100] m, Hs U[1,4] m, 200 modes, FP64",
                   "units_per_step_per_gpu": units},
        "eager": {"value": units * args.steps / eager_s, "ms_per_step": 1e3 * eager_s / args.steps,
                  "kernel_launches_per_step": int(launches)},
        "lanes": {"chosen": lanes, "autotune_seconds": t_tune,
                  "one_lane_value": units * args.steps / serial_s},
        "tiles": {"plans_tuned_off_default": tuned, "plans": len(runner.staged),
                  "autotune_seconds": t_tiles,
                  "builtin_shapes_value": units * args.steps / untuned_s},
        "kernel_shares": [{"name": r["name"], "launches": r["launches"],
                           "share": round(r["ms_total"] / ktot, 4)} for r in kstats[:10]],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_config4(args, rank: int, world: int, local_rank: int) -> None:
    """Adjoint fit: the gradient of ||eta11 + eta22 + eta33 - eta_obs||^2 with
    respect to the a, b of 2048 modes on a 512^2 grid (h=25 m, Hs=2.5 m,
    eta22 rank 6, order 3 GL4/GL4), eta_obs from a held-out seed plus
    N(0, 0.01 m) noise.  A step = one forward + one backward through the
    torch.autograd.Function (the backward is one gl_adjoint_execute pass).
    Each rank fits its own sea state (seed = rank): no collective."""
    import numpy as np
    import torch

    from gl_engine import _lib, seastate
    from gl_engine.adjoint import EtaSurfaceModel, eta_surface

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    st = seastate.config4(seed=rank)
    held = seastate.config4(seed=1000 + rank)
    model = EtaSurfaceModel(st.kx, st.ky, depth=st.depth, lx=st.lx, ly=st.ly, nx=st.nx, ny=st.ny,
                            times=[0.0], order=3, eta22_rank=6, device=device)
    gen = torch.Generator(device="cpu").manual_seed(rank)
    obs = model.eta(torch.tensor(held.a, device=device), torch.tensor(held.b, device=device))
    obs = obs + 0.01 * torch.randn(obs.shape, generator=gen, dtype=torch.float64).to(device)
    a = torch.tensor(st.a, device=device, requires_grad=True)
    b = torch.tensor(st.b, device=device, requires_grad=True)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)

    def step():
        a.grad = None
        b.grad = None
        loss = ((eta_surface(a, b, model) - obs) ** 2).sum()
        loss.backward()
        return loss

    def timed(fn, n):
        tot = 0.0
        for _ in range(n):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
        return tot

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = _lib.launch_count()
    with ClockSampler(local_rank) as clk:
        t_step = timed(step, args.steps)
    launches = (_lib.launch_count() - launches0) // max(args.steps, 1)
    ad, bd = a.detach(), b.detach()
    resid = 2.0 * (model.eta(ad, bd) - obs)
    t_fwd = timed(lambda: model.eta(ad, bd), args.steps)
    t_bwd = timed(lambda: model.vjp(ad, bd, resid), args.steps)
    if world > 1:
        import torch.distributed as dist

        tt = torch.tensor([t_step, t_fwd, t_bwd], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_step, t_fwd, t_bwd = (float(v) for v in tt)
    # end to end: host amplitudes in, host gradients out, every step
    a_host = torch.from_numpy(st.a.copy()).pin_memory()
    b_host = torch.from_numpy(st.b.copy()).pin_memory()
    ga_host = torch.empty_like(a_host).pin_memory()
    gb_host = torch.empty_like(b_host).pin_memory()

    def e2e_step():
        with torch.no_grad():
            a.copy_(a_host, non_blocking=True)
            b.copy_(b_host, non_blocking=True)
        step()
        ga_host.copy_(a.grad, non_blocking=True)
        gb_host.copy_(b.grad, non_blocking=True)
        torch.cuda.synchronize()

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e2e = time.perf_counter() - t0
    # a short fit: Adam on the amplitudes from the engine's gradient
    fit_a = torch.tensor(st.a, device=device, requires_grad=True)
    fit_b = torch.tensor(st.b, device=device, requires_grad=True)
    opt = torch.optim.Adam([fit_a, fit_b], lr=2e-3)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        loss = ((eta_surface(fit_a, fit_b, model) - obs) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    n = args.steps
    line = {
        "metric": "config-4 adjoint fit: gradients/s of ||eta11+eta22+eta33 - eta_obs||^2 wrt a,b",
        "value": world * n / t_step, "unit": "gradients/s", "n_gpus": world, "steps": n,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_step / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded JONSWAP sea state; eta_obs from a held-out seed + N(0, 0.01 m))",
        "config": {"workload": "order-3 eta11+eta22(rank 6)+eta33 (GL4/GL4), 512^2 grid, L=512 m, "
                               "h=25 m, Hs=2.5 m, 2048 modes; step = forward + backward",
                   "l2": "flushed between timed steps (256 MiB write outside the events)",
                   "parallelism": f"one sea state per rank over {world} rank(s), no collective"},
        "forward_ms": 1e3 * t_fwd / n, "backward_ms": 1e3 * t_bwd / n,
        "backward_over_forward": t_bwd / t_fwd,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "e2e": {"value": world * n / t_e2e, "unit": "gradients/s",
                "h2d_bytes_per_step": int(2 * 8 * st.a.size), "d2h_bytes_per_step": int(2 * 8 * st.a.size)},
        "fit_demo": {"optimizer": "Adam lr 2e-3", "steps": len(losses), "loss_first": losses[0],
                     "loss_last": losses[-1]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import gl_torch as GT

        k = np.hypot(st.kx, st.ky)
        omega = np.sqrt(9.81 * k * np.tanh(st.depth * k))
        ac = torch.tensor(st.a, requires_grad=True)
        bc = torch.tensor(st.b, requires_grad=True)
        t0 = time.perf_counter()
        eta = GT.eta_surface(ac, bc, kx=st.kx, ky=st.ky, omega=omega, depth=st.depth, lx=st.lx,
                             ly=st.ly, nx=st.nx, ny=st.ny, t=0.0, eta22_rank=6)
        ((eta - obs[0].cpu()) ** 2).sum().backward()
        t_cpu = time.perf_counter() - t0
        ga, gb = model.vjp(ad, bd, resid)
        g_gpu = np.r_[ga.cpu().numpy(), gb.cpu().numpy()]
        g_cpu = np.r_[ac.grad.numpy(), bc.grad.numpy()]
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "gradients/s",
                                "cores": torch.get_num_threads(), "kind": "port",
                                "sample": "one full gradient: torch.autograd through the FP64 oracle "
                                          "transliteration (oracle/gl_torch.py) on the host CPU"}
        line["parity_vs_oracle"] = {
            "gradient_rel_l2": float(np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu))}
    if rank == 0:
        print(json.dumps(line), flush=True)


# published order-4 timings of the reference (paper/order4/data/runtime/
# eta44_runtime_figure_data.csv; C++ on 32 cores of a Xeon Silver 4214, 512^2)
PUBLISHED_GL_N1500_S = {6: 11.31350016, 8: 20.21097216, 10: 35.332300544}
PUBLISHED_WIT_S = {50: 0.765824, 100: 6.76152, 200: 96.4575, 300: 476.281, 400: 1491.09,
                   500: 3614.69, 600: 7502.55, 800: 21856.765945183}


def _eta44_timed(spec, n, dk, rank_gl, steps, device):
    """Device seconds per eta44 field of one spectrum at GL ``rank_gl``, its
    launches, status and plan grids."""
    import torch

    from gl_engine import _lib
    from gl_engine import eta44 as E44

    box = E44._box(spec)
    desc = _lib.Eta44Desc(n=n, dk=dk, depth=1.0, peak_depth=1.0, rank=rank_gl, nodes=None,
                          weights=None, box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3],
                          max_units=1, output=_lib.OUT_COMPLEX)
    plan = E44.Eta44Plan(desc, device)
    stream = torch.cuda.current_stream(device)
    d_spec = torch.view_as_real(torch.from_numpy(spec).to(device))
    out = torch.empty((1, 1, n, n), dtype=torch.complex128, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)

    def run():
        plan.execute(1, d_spec, _lib.SPECTRA_FULL, out, status, stream.cuda_stream)

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = _lib.launch_count()
    e0.record(stream)
    for _ in range(steps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    return {"seconds": e0.elapsed_time(e1) / 1e3 / steps,
            "gpu_launches": int((_lib.launch_count() - launches0) // steps),
            "status": int(status.item()), "transforms_per_field": plan.info.transforms_per_unit,
            "product_grid": [plan.info.ncy, plan.info.ncx]}


def run_config5(args, rank: int, world: int, local_rank: int) -> None:
    """Order 4.  Headline: the dimensionless 1024^2 case of 1024 modes (g = h
    = 1, peak kh 1.5, steepness 0.08; seastate.config5_case) at GL6/8/10 with
    the FP64 quadrature sum, cross-checked against the WIT quartet sum over
    its 128 largest modes (C(131, 4) = 11.7 M quartets) -- GL-vs-WIT raw
    relative L2 per rank for peak kh 0.8, 1.5 and 3, and the GPU WIT against
    the reference's own WIT C++ (oracle/_ref/wit_eta44, built from its
    sources) on the kh 1.5 subset.  Also the reference's runtime ladder
    (512^2, dk = 0.1: the DIR4IN01 inputs behind its published timings)
    against the published C++ wall times.  Rank 0 only."""
    import numpy as np
    import torch

    from gl_engine import seastate, wit
    from gl_engine import eta44 as E44

    if rank != 0:
        return
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    steps = max(1, min(args.steps, 3))

    def l2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    # --- the stated 1024^2 / 1024-mode case
    case = seastate.config5_case(peak_kh=1.5, steepness=0.08, modes=1024, n=1024, seed=0)
    n = case.nx
    spec = E44.spectrum_from_modes(case.modes, case.amplitudes[0], n, case.depth)
    stated = {str(r): _eta44_timed(spec, n, case.dkx, r, steps, device) for r in (6, 8, 10)}
    t0 = time.perf_counter()
    E44.eta44(spec, dk=case.dkx, depth=1.0, peak_depth=1.0, rank=10, device=device)
    e2e_s = time.perf_counter() - t0
    # --- GL vs WIT on the 128 largest modes, three peak kh
    cross = {}
    ref_bin = ROOT / "oracle" / "_ref" / "wit_eta44"
    for kh in (0.8, 1.5, 3.0):
        full = seastate.config5_case(peak_kh=kh, steepness=0.08, modes=1024, n=n, seed=0)
        sub = seastate.largest_modes(full, 128)
        s_sub = E44.spectrum_from_modes(sub.modes, sub.amplitudes[0], n, sub.depth)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        w = wit.wit_sector(sub, 44, device=device)
        wit_s = time.perf_counter() - t0
        wit_eta = np.real(np.fft.ifft2(w.fields["eta"][0] * n * n))
        row = {"wit_quartets": int(w.stats["candidates"]), "wit_kept": int(w.stats["kept"]),
               "wit_seconds": wit_s, "gl_vs_wit_raw_rel_l2_pct": {}}
        for r in (6, 8, 10):
            gl = np.real(E44.eta44(s_sub, dk=sub.dkx, depth=1.0, peak_depth=1.0, rank=r,
                                   device=device))
            row["gl_vs_wit_raw_rel_l2_pct"][str(r)] = 100 * l2(gl, wit_eta)
        if kh == 1.5 and ref_bin.exists() and not args.no_cpu_baseline:
            with tempfile.TemporaryDirectory() as td:
                wit.write_dir4in(Path(td) / "in.bin", sub)
                t0 = time.perf_counter()
                subprocess.run([str(ref_bin), str(Path(td) / "in.bin"), str(Path(td) / "o.bin"),
                                "--sector", "44"], check=True, capture_output=True,
                               env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count())))
                row["reference_wit_seconds"] = time.perf_counter() - t0
                ref = wit.read_dir4out(Path(td) / "o.bin")
                row["wit_vs_reference_rel_l2"] = {
                    f: l2(w.fields[f][0], ref.fields[f][0]) for f in ("eta", "psi")}
                row["reference_wit_cores"] = os.cpu_count()
        cross[str(kh)] = row
    # --- the reference's runtime ladder against its published timings
    gold = ROOT / "tests" / "golden" / "runtime"
    inp = wit.read_dir4in(gold / "n1500.bin")
    spec_l = E44.spectrum_from_modes(inp.modes, inp.amplitudes[0], inp.nx, inp.depth)
    ladder = {}
    for r in (6, 8, 10):
        g = _eta44_timed(spec_l, inp.nx, inp.dkx, r, steps, device)
        g["published_cpp_seconds"] = PUBLISHED_GL_N1500_S[r]
        g["speedup_vs_published"] = PUBLISHED_GL_N1500_S[r] / g["seconds"]
        ladder[f"gl{r}_n1500"] = g
    for m in (50, 100, 200, 300, 400):
        wi = wit.read_dir4in(gold / f"n{m:04d}.bin")
        wit.wit_sector(wi, 44, device=device)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = wit.wit_sector(wi, 44, device=device)
        sec = time.perf_counter() - t0
        ladder[f"wit_n{m:04d}"] = {"seconds": sec, "quartets": int(res.stats["candidates"]),
                                   "published_cpp_seconds": PUBLISHED_WIT_S[m],
                                   "speedup_vs_published": PUBLISHED_WIT_S[m] / sec}
    cpu = None
    if ref_bin.exists() and not args.no_cpu_baseline and "reference_wit_seconds" in cross["1.5"]:
        cs = cross["1.5"]["reference_wit_seconds"]
        cpu = {"value": 1.0 / cs, "unit": "WIT fields/s (128 modes, 1024^2)", "cores": os.cpu_count(),
               "kind": "reference",
               "sample": "the reference's WIT C++ (oracle/_ref/wit_eta44, OpenMP on all host cores) on "
                         f"the 128 largest modes of the kh 1.5 case: {cs:.2f} s; GPU "
                         f"{cross['1.5']['wit_seconds']:.3f} s"}
    sec10 = stated["10"]["seconds"]
    value = 1.0 / sec10
    line = {
        "metric": "order-4 eta44 GL10 fields/s, 1024^2, 1024 modes (g=h=1, peak kh 1.5, steepness 0.08)",
        "value": value, "unit": "fields/s", "n_gpus": 1, "steps": steps,
        "warmup": 1, "ms_per_step": 1e3 * sec10, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded dimensionless sea states (seastate.config5_case); the runtime "
                "ladder uses the reference's own DIR4IN01 inputs (tests/golden/runtime)",
        "config": {"workload": "eta44 GL6/8/10 (three nested GL levels, FP64 quadrature sum) on "
                               "1024^2 with 1024 modes; WIT sector 44 over the 128 largest modes "
                               "for peak kh 0.8/1.5/3",
                   "inputs_vs_l2": "single field per step; inputs above L2 not applicable"},
        "gl": stated,
        "wit_cross_check": cross,
        "runtime_ladder": ladder,
        "gpu_launches": stated["10"]["gpu_launches"],
        "e2e": {"value": 1.0 / e2e_s, "unit": "fields/s", "h2d_bytes_per_step": int(spec.nbytes),
                "d2h_bytes_per_step": int(n * n * 16)},
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def _timeseries_record(n: int, dt: float, seed: int = 0, hs: float = 2.0, tp: float = 8.0):
    """Seeded single-direction JONSWAP record (gamma 3.3) of n samples."""
    import numpy as np

    rng = np.random.default_rng(seed)
    w = 2 * np.pi * np.fft.rfftfreq(n, dt)[1:]
    wp = 2 * np.pi / tp
    sig = np.where(w <= wp, 0.07, 0.09)
    spec = 9.81**2 / w**5 * np.exp(-1.25 * (wp / w) ** 4) * 3.3 ** np.exp(-(w - wp) ** 2 / (2 * sig**2 * wp**2))
    spec = spec * (hs**2 / 16) / np.sum(spec * (w[1] - w[0]))
    amp = np.sqrt(2 * spec * (w[1] - w[0]))
    phase = rng.uniform(0, 2 * np.pi, amp.size)
    t = np.arange(n) * dt
    eta = np.sum(amp[:, None] * np.cos(w[:, None] * t[None, :] + phase[:, None]), axis=0)
    return eta, t


def run_timeseries(args, rank: int, world: int, local_rank: int) -> None:
    """Single-direction time path (the reference's modal_time.py): a seeded
    1024-sample JONSWAP record (dt 0.25 s, h 20 m, Hs 2 m, Tp 8 s), order 3 at
    GL8 with eta20, through the reference's default modal ladder (2048 ..
    65536 q-nodes, tolerance 1e-3).  Rank 0 only; the CPU baseline is the
    oracle port on the first two ladder levels."""
    import numpy as np
    import torch

    from gl_engine import _lib
    from gl_engine import modal

    if rank != 0:
        return
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    eta1, t = _timeseries_record(1024, 0.25)
    kw = dict(depth=20.0, order=3, quadrature_rank=8, include_eta20=True)
    modal.reconstruct_unidirectional_timeseries(eta1, t, modal_points=(2048, 4096), **kw)  # warm-up
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 5))
    launches0 = _lib.launch_count()
    t0 = time.perf_counter()
    for _ in range(steps):
        res = modal.reconstruct_unidirectional_timeseries(eta1, t, **kw)
    torch.cuda.synchronize()
    sec = (time.perf_counter() - t0) / steps
    launches = (_lib.launch_count() - launches0) // steps
    t0 = time.perf_counter()
    short = modal.reconstruct_unidirectional_timeseries(eta1, t, modal_points=(2048, 4096), **kw)
    gpu_short = time.perf_counter() - t0
    line = {
        "metric": "single-direction time series (modal GL, order 3 + eta20) records/s",
        "value": 1.0 / sec, "unit": "records/s", "n_gpus": 1, "steps": steps, "warmup": 1,
        "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded 1024-sample JONSWAP record)",
        "config": {"workload": "1024 samples, dt 0.25 s, h 20 m, order 3, GL8, eta20 rank 16 on 128x16, "
                               "modal ladder 2048..65536 to tolerance 1e-3 (e2e: host record in, "
                               "host series out)"},
        "levels": [lv["modal_points"] for lv in res.audit["levels"]],
        "converged": bool(res.audit["converged"]), "gpu_launches": int(launches),
        "e2e": {"value": 1.0 / sec, "unit": "records/s", "h2d_bytes_per_step": int(eta1.nbytes),
                "d2h_bytes_per_step": int(4 * eta1.nbytes)},
    }
    if not args.no_cpu_baseline:
        from oracle import gl_modal as M

        t0 = time.perf_counter()
        _, c, _ = M.modal_timeseries(eta1, t, modal_points=(2048, 4096), **kw)
        cpu = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / cpu, "unit": "records/s (ladder 2048, 4096)", "cores": 1,
                                "kind": "port",
                                "sample": f"the first two ladder levels + eta20 by the NumPy oracle: "
                                          f"{cpu:.2f} s; GPU on the same sample {gpu_short:.3f} s"}
        line["parity_vs_oracle"] = {k: float(np.linalg.norm(short.components[k] - c[k])
                                             / np.linalg.norm(c[k])) for k in ("eta22", "eta33", "eta20")}
    print(json.dumps(line), flush=True)


def _relaunch_ranks(n: int) -> None:
    """``--gpus N`` without a launcher: start N ranks of this script on this
    node through torch.distributed.run (one process per GPU, 127.0.0.1
    rendezvous), which then sets RANK / LOCAL_RANK / WORLD_SIZE."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__),
           *sys.argv[1:]]
    sys.stdout.flush()
    os.execv(sys.executable, cmd)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--units", type=int, default=16, help="units per step per GPU")
    ap.add_argument("--group", type=int, default=0, help="units per engine launch group")
    ap.add_argument("--lanes", type=int, default=2,
                    help="concurrent lanes of the engine plan (groups of units / lanes units)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain-gpu", action="store_true",
                    help="skip the plain single-field cuFFT comparison leg")
    ap.add_argument("--workload", choices=["config2", "config3", "config4", "config5", "timeseries"],
                    default="config2",
                    help="config2: the headline order-3 1024^2 workload; config3: uneven batch; "
                         "config4: adjoint fit; config5: order 4 (eta44 GL, WIT) on the reference's "
                         "runtime inputs; timeseries: the single-direction modal time path")
    ap.add_argument("--states", type=int, default=64, help="config3: sea states per GPU")
    ap.add_argument("--launch-check", action="store_true",
                    help="print each rank's RANK / WORLD_SIZE as JSON and exit (checks the "
                         "multi-rank launch without touching a GPU)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        _relaunch_ranks(args.gpus)  # does not return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world != max(1, args.gpus):
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
    if args.launch_check:
        print(json.dumps({"rank": rank, "local_rank": local_rank, "world": world}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "config3":
            run_config3(args, rank, world, local_rank)
        elif args.workload == "config4":
            run_config4(args, rank, world, local_rank)
        elif args.workload == "config5":
            run_config5(args, rank, world, local_rank)
        elif args.workload == "timeseries":
            run_timeseries(args, rank, world, local_rank)
        else:
            run_engine(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
