"""Uneven batches: many sea states of different grids, orders, ranks and
depths evaluated as one captured CUDA graph.

Each sea state gets its own plan (grid, box, ranks).  The states are dealt
to ``lanes`` concurrent streams (longest-first onto the least-loaded lane,
by estimated transform work); every lane has its own device workspace and
runs its states one after another, and the lanes run side by side, so the
small 128^2 / 256^2 states fill the SMs next to the large ones instead of
leaving them idle.  Every input is staged on the device before capture, and
the whole batch -- one deposit and one gl_execute per sea state, the lanes as
parallel branches between one fork and one join -- is captured once and
replayed.  Replays skip the host entirely: no Python, no argument marshalling,
no launch latency between the ~40 kernels of each sea state.

``autotune_group`` times the units-per-launch group size of a plan on the
device, ``autotune_tiles`` the launch shapes of its transform kernels
(transform groups per row block of the pair and triple stages, columns per
column block: ``Plan.set_tuning``), and ``autotune_lanes`` the lane count of
a batch; all cache the fastest choice in memory (and in a JSON file when
``GL_AUTOTUNE_CACHE`` names one).
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, api, seastate


@dataclass
class BatchItem:
    coeffs: api.GLCoefficients
    lx: float
    ly: float
    nx: int
    ny: int
    times: np.ndarray
    components: tuple = ()
    inner_rank: int = 4
    outer_rank: int = 4
    group: int = 0  # units per launch (0: all snapshots)


@dataclass
class _Staged:
    item: BatchItem
    plan: api.Plan
    dep: api.ModeDeposit
    tensors: dict = field(default_factory=dict)


def _work_estimate(plan: api.Plan, n_units: int) -> float:
    """Transform work of one sea state: transforms per unit x the product grid."""
    info = plan.info
    return float(info.transforms_per_unit) * info.ncx * info.ncy * max(1, n_units)


class BatchRunner:
    """Stage, capture and replay an uneven batch of sea states on one GPU."""

    def __init__(self, items: list[BatchItem], *, device=None, output: str = "real",
                 lanes: int = 4, tiles: str | None = None):
        self.device = torch.device(device if device is not None else "cuda")
        self.output = _lib.OUT_REAL if output == "real" else _lib.OUT_COMPLEX
        self.items = items
        self.staged: list[_Staged] = []
        self.graph = None
        with torch.cuda.device(self.device):
            for it in items:
                mask = api._components_for(it.coeffs.order, it.components or None)
                dep = api.prepare_deposit(it.coeffs, it.lx, it.ly, it.nx, it.ny)
                n = int(np.size(it.times))
                plan = api.get_plan(nx=it.nx, ny=it.ny, lx=it.lx, ly=it.ly, depth=it.coeffs.h,
                                    gravity=it.coeffs.g, order=it.coeffs.order, components=mask,
                                    eta22_rank=int(it.coeffs.options["eta22_rank"]),
                                    allow_below=it.coeffs.options["allow_below_model_parent_domain"],
                                    box=dep.box, grid=_lib.GRID_COMPACT,
                                    max_units=it.group or n, output=self.output,
                                    device=self.device, inner_rank=it.inner_rank,
                                    outer_rank=it.outer_rank)
                self.staged.append(_Staged(it, plan, dep))
            if tiles == "auto":  # tuned launch shapes per plan shape (cached)
                for st in self.staged:
                    st.plan.set_tuning(*autotune_tiles(st.item, device=self.device))
            # lanes: longest first onto the least-loaded lane
            k = max(1, min(int(lanes), len(self.staged)))
            load = [0.0] * k
            self.lane_of = [0] * len(self.staged)
            order = sorted(range(len(self.staged)), key=lambda i: -_work_estimate(
                self.staged[i].plan, int(np.size(self.staged[i].item.times))))
            for i in order:
                lane = int(np.argmin(load))
                self.lane_of[i] = lane
                load[lane] += _work_estimate(self.staged[i].plan, int(np.size(self.staged[i].item.times)))
            self.lanes = k
            self.workspaces = []
            for lane in range(k):
                ws = max([s.plan.workspace_bytes for i, s in enumerate(self.staged)
                          if self.lane_of[i] == lane] or [0])
                buf = torch.empty(ws + 256, dtype=torch.uint8, device=self.device)
                self.workspaces.append((buf, (buf.data_ptr() + 255) & ~255, ws))
            self.streams = [torch.cuda.Stream(self.device) for _ in range(k)]
            dtype = torch.float64 if self.output == _lib.OUT_REAL else torch.complex128
            for s in self.staged:
                dev = self.device
                t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
                n = int(np.size(s.item.times))
                w, h = s.dep.box[2], s.dep.box[3]
                s.tensors = {
                    "seg_off": t(s.dep.seg_offsets, torch.int32),
                    "seg_bin": t(s.dep.seg_bins, torch.int32),
                    "ab": t(s.dep.ab, torch.float64),
                    "omega": t(s.dep.omega, torch.float64),
                    "times": t(np.asarray(s.item.times, dtype=float), torch.float64),
                    "spectra": torch.empty((n, h, w, 2), dtype=torch.float64, device=dev),
                    "out": torch.empty((n, s.plan.info.n_components, s.item.ny, s.item.nx),
                                       dtype=dtype, device=dev),
                    "status": torch.zeros(n, dtype=torch.int32, device=dev),
                }
        self.units = sum(int(np.size(s.item.times)) for s in self.staged)

    def _enqueue_lane(self, lane: int, stream: int) -> None:
        lib = _lib.load()
        import ctypes as C

        _, ws_ptr, ws_bytes = self.workspaces[lane]
        for i, s in enumerate(self.staged):
            if self.lane_of[i] != lane:
                continue
            t = s.tensors
            n = int(t["times"].numel())
            s.plan.deposit(n, t["seg_off"], t["seg_bin"], t["ab"], t["omega"], t["times"],
                           t["spectra"], stream)
            api._engine_call(lib.gl_execute(
                s.plan.handle, n, C.c_void_p(t["spectra"].data_ptr()), _lib.SPECTRA_BOX,
                C.c_void_p(t["out"].data_ptr()), C.c_void_p(ws_ptr), C.c_size_t(ws_bytes),
                C.c_void_p(t["status"].data_ptr()), C.c_void_p(stream)))

    def _enqueue(self, main: torch.cuda.Stream) -> None:
        """Fork from ``main`` onto the lane streams and join back (in a
        capture this makes the lanes parallel branches of one graph)."""
        fork = torch.cuda.Event()
        fork.record(main)
        for lane, ls in enumerate(self.streams):
            ls.wait_event(fork)
            self._enqueue_lane(lane, ls.cuda_stream)
            done = torch.cuda.Event()
            done.record(ls)
            main.wait_event(done)

    def run_eager(self) -> None:
        with torch.cuda.device(self.device):
            self._enqueue(torch.cuda.current_stream(self.device))

    def capture(self) -> None:
        """Warm up once (kernel attributes, caches), then capture the batch."""
        with torch.cuda.device(self.device):
            self.run_eager()
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream(self.device)
            with torch.cuda.stream(side):
                with torch.cuda.graph(g, stream=side):
                    self._enqueue(side)
            self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def check(self) -> None:
        for s in self.staged:
            st = s.tensors["status"].cpu().numpy()
            if np.any(st != 0):
                raise api._status_error(int(st[st != 0][0]))

    def outputs(self):
        return [(s.item, [api.COMP_NAMES[c] for c in s.plan.component_ids], s.tensors["out"])
                for s in self.staged]


def config3_items(n_states: int = 64, snapshots: int = 8, seed0: int = 0, modes: int = 200,
                  grids=(128, 256, 512, 1024)) -> list[BatchItem]:
    """The uneven batch: seeds seed0.., grids from {128..1024}^2, orders 2-3,
    ranks {2,4,6,8}, snapshots t ~ U[0,60] s, h ~ U[10,100] m, Hs ~ U[1,4] m,
    L = N * 2 m.  Rank 2 is not an order-3 rank, so the drawn rank sets
    eta22_rank and the order-3 (inner, outer) ranks are (r, r) for r in
    {4, 6, 8} and (4, 4) for r = 2."""
    rng = np.random.default_rng(seed0 + 1234)
    out = []
    for k in range(n_states):
        n = int(rng.choice(grids))
        order = int(rng.integers(2, 4))
        rank = int(rng.choice([2, 4, 6, 8]))
        depth = float(rng.uniform(10.0, 100.0))
        hs = float(rng.uniform(1.0, 4.0))
        times = rng.uniform(0.0, 60.0, snapshots)
        st = seastate.jonswap_sea_state(n=n, length=2.0 * n, depth=depth, hs=hs, tp=10.0,
                                        modes=modes, seed=seed0 + k, order=order)
        coeffs = api.gl_spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx,
                                              st.ky, 0.0, 0.0, {"eta22_rank": rank})
        r3 = rank if rank in (4, 6, 8) else 4
        comps = ("eta22", "psi22") if order == 2 else ("eta33", "psi33")
        out.append(BatchItem(coeffs=coeffs, lx=st.lx, ly=st.ly, nx=n, ny=n, times=times,
                             components=comps, inner_rank=r3, outer_rank=r3))
    return out


_TUNE: dict = {}


def _tune_cache_load() -> None:
    path = os.environ.get("GL_AUTOTUNE_CACHE")
    if path and not _TUNE and os.path.exists(path):
        for k, v in json.load(open(path)).items():
            _TUNE[k] = v


def _tune_cache_store() -> None:
    path = os.environ.get("GL_AUTOTUNE_CACHE")
    if path:
        with open(path, "w") as f:
            json.dump(_TUNE, f)


def autotune_lanes(items: list[BatchItem], *, candidates=(1, 2, 4, 8), device=None,
                   repeats: int = 2) -> int:
    """Concurrent lanes that minimise the device time of this batch's replay."""
    key = repr(("lanes", tuple(sorted((it.nx, it.coeffs.order, it.inner_rank,
                                       int(it.coeffs.options["eta22_rank"]),
                                       int(np.size(it.times))) for it in items)), tuple(candidates)))
    _tune_cache_load()
    if key in _TUNE:
        return int(_TUNE[key])
    best, best_t = None, float("inf")
    for k in candidates:
        runner = BatchRunner(items, device=device, lanes=k)
        runner.capture()
        runner.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            runner.replay()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        del runner
        if t < best_t:
            best, best_t = k, t
    _TUNE[key] = best
    _tune_cache_store()
    return int(best)


def autotune_group(item: BatchItem, *, candidates=(1, 2, 4, 8, 16), device=None,
                   repeats: int = 3) -> int:
    """Units per launch that minimise device time for this item's plan shape."""
    key = (item.nx, item.ny, item.coeffs.order, item.inner_rank, item.outer_rank,
           api.prepare_deposit(item.coeffs, item.lx, item.ly, item.nx, item.ny).box,
           tuple(item.components))
    _tune_cache_load()
    skey = repr(key)
    if skey in _TUNE:
        return int(_TUNE[skey])
    n = int(np.size(item.times))
    best, best_t = None, float("inf")
    for g in candidates:
        if g > n:
            continue
        trial = BatchItem(**{**item.__dict__, "group": g})
        runner = BatchRunner([trial], device=device, lanes=1)
        runner.run_eager()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            runner.run_eager()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        if t < best_t:
            best, best_t = g, t
    _TUNE[skey] = best
    _tune_cache_store()
    return int(best)


TILE_CANDIDATES = {"pair_row_groups": (0, 4, 16), "triple_row_groups": (0, 8, 16),
                   "col_block_columns": (0, 8, 4)}


def autotune_tiles(item: BatchItem, *, device=None, repeats: int = 3) -> tuple:
    """Launch shapes (pair row groups, triple row groups, columns per column
    block) that minimise one eager run of this item's plan, by coordinate
    descent from the built-in choices (0) over ``TILE_CANDIDATES``; the plan's
    shape -- grid, order, ranks, box -- is the cache key."""
    dep = api.prepare_deposit(item.coeffs, item.lx, item.ly, item.nx, item.ny)
    key = repr(("tiles", item.nx, item.ny, item.coeffs.order, item.inner_rank, item.outer_rank,
                int(item.coeffs.options["eta22_rank"]), dep.box, tuple(item.components),
                int(np.size(item.times)), item.group))
    _tune_cache_load()
    if key in _TUNE:
        return tuple(_TUNE[key])
    runner = BatchRunner([item], device=device, lanes=1)
    plan = runner.staged[0].plan

    def timed(cfg):
        plan.set_tuning(*cfg)
        runner.run_eager()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            runner.run_eager()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    best = [0, 0, 0]
    best_t = timed(tuple(best))
    for k, name in enumerate(("pair_row_groups", "triple_row_groups", "col_block_columns")):
        if name == "triple_row_groups" and item.coeffs.order < 3:
            continue
        for v in TILE_CANDIDATES[name]:
            if v == best[k]:
                continue
            cfg = list(best)
            cfg[k] = v
            t = timed(tuple(cfg))
            if t < best_t:
                best, best_t = cfg, t
    plan.set_tuning(0, 0, 0)
    _TUNE[key] = list(best)
    _tune_cache_store()
    return tuple(best)

