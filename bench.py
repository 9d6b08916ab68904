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
  ``e2e`` times the public API with host inputs and a device->host read of
  the real fields each step.
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
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------


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

    # ---- per-kernel breakdown (separate profiled pass, events per launch)
    _lib.profile_begin()
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    kstats = _lib.profile_end()
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
        host = torch.empty((U, 2, st.ny, st.nx), dtype=torch.float64, pin_memory=True)
        e2e_out = torch.empty_like(out)
        h2d = dep.ab.nbytes + dep.omega.nbytes + dep.seg_offsets.nbytes + dep.seg_bins.nbytes + \
            times.nbytes
        d2h = host.numel() * 8

        def e2e_step():
            res = api.surface_batch_device(coeffs, st.lx, st.ly, st.nx, st.ny, times,
                                           components=["eta33", "psi33"], output="real",
                                           device=device, max_units=args.group or U,
                                           out=e2e_out, check=False)
            host.copy_(res.fields, non_blocking=True)
            torch.cuda.current_stream(device).synchronize()

        for _ in range(2):
            e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=device)
        if world > 1:
            dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
        e2e = {"value": U * args.steps * world / float(e2e_s.item()), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded JONSWAP + cos^2s sea state; no dataset)",
        "config": workload_config(U, world, [plan.info.ncy, plan.info.ncx]),
        "roofline": roofline, "accounting": accounting, "clocks": clocks,
        "gpu_launches": int(launches), "e2e": e2e,
    }
    if world == 1 and not args.no_cpu_baseline:
        base, (e_ref, p_ref) = cpu_baseline_sample()
        line["cpu_baseline"] = base
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        line["parity_vs_oracle"] = {"eta33_rel_l2": rel(first[0], e_ref.real),
                                    "psi33_rel_l2": rel(first[1], p_ref.real)}
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
    runner = batch.BatchRunner(items, device=device)
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
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--units", type=int, default=16, help="units per step per GPU")
    ap.add_argument("--group", type=int, default=0, help="units per engine launch group")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["config2", "config3"], default="config2",
                    help="config2: the headline order-3 1024^2 workload; config3: uneven batch")
    ap.add_argument("--states", type=int, default=64, help="config3: sea states per GPU")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
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
        else:
            run_engine(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
