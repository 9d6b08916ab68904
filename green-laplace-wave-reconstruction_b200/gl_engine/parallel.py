"""Multi-GPU orchestration (one process per GPU, torch.distributed).

The GL path shards in two ways:

* independent units (sea states x snapshots): each rank evaluates its own
  contiguous share, no collective on the data path (``shard_units``);
* the WIT quartet sum: the sector's candidate quartets are split into
  contiguous, equal-count index ranges (every candidate costs about the
  same: one 15-subset recursion), each rank sums its share into zeroed field
  planes, and one all-reduce sums the 5 planes (``wit_sharded`` /
  ``wit_sector_distributed``): the device form of the reference's
  per-thread accumulators and serial merge
  (``paper/order4/cpp/directional_eta4_openmp.cpp:734-745``);
* one large eta44 field: the GL outer nodes are split across ranks, each rank
  accumulates a partial order-4 spectrum on the small quartic box, one
  all-reduce (NCCL over NVLink on GPUs) sums the partials, and the final
  roundoff floor and inverse transform run once (``eta44_sharded``).  This is
  the device analogue of the reference's process split
  (``paper/order4/run_gl_split.sh:31-38``) and its file merge
  (``paper/order4/cpp/merge_eta44_outer.cpp:12``), except that the partial
  spectra are summed before the final floor, so the sharded result equals the
  single-GPU one up to summation order.
"""

from __future__ import annotations

import ctypes as C
from typing import Callable

import numpy as np


def split_range(count: int, rank: int, world: int) -> tuple[int, int]:
    """Balanced contiguous [begin, end) share of ``count`` items for ``rank``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard_units(n_units: int, rank: int, world: int) -> slice:
    b, e = split_range(n_units, rank, world)
    return slice(b, e)


def eta44_sharded(compute_partial: Callable[[int, int], object], reduce_sum: Callable[[object], object],
                  finalize: Callable[[object], object], zeros: Callable[[], object], rank: int,
                  rank_count: int, world: int):
    """Outer-node sharding driver, independent of the backend.

    ``compute_partial(begin, end)`` returns this rank's partial spectrum,
    ``reduce_sum(x)`` sums it over ranks (in place or returned), ``finalize``
    turns the sum into fields.  Ranks without nodes contribute ``zeros()``.
    """
    b, e = split_range(rank_count, rank, world)
    part = compute_partial(b, e) if b < e else zeros()
    total = reduce_sum(part)
    return finalize(part if total is None else total)


STAT_SUMS = ("candidates", "kept", "near", "strict_zero_output", "strict_zero_intermediate")
STAT_MAXES = ("max_residual", "max_strict_zero_source")
STAT_MINS = ("min_detuning",)


def combine_wit_stats(parts: list[dict]) -> dict:
    """Statistics of the whole sum from those of its shares."""
    out = {k: sum(int(p[k]) for p in parts) for k in STAT_SUMS}
    out.update({k: max(float(p[k]) for p in parts) for k in STAT_MAXES})
    out.update({k: min(float(p[k]) for p in parts) for k in STAT_MINS})
    return out


def wit_sharded(compute_range: Callable[[int, int], tuple], reduce_sum: Callable[[object], object],
                gather_stats: Callable[[dict], list], count: int, rank: int, world: int):
    """Quartet-range sharding driver, independent of the backend.

    ``compute_range(begin, end)`` returns (fields, stats) of this rank's
    share of the ``count`` candidates (zero fields for an empty share),
    ``reduce_sum(fields)`` sums the field planes over ranks (in place or
    returned) and ``gather_stats(stats)`` returns every rank's statistics.
    Every rank returns the full fields and the combined statistics."""
    b, e = split_range(count, rank, world)
    fields, stats = compute_range(b, e)
    total = reduce_sum(fields)
    return (fields if total is None else total), combine_wit_stats(gather_stats(stats))


def wit_sector_distributed(inp, sector: int = 44, *, group=None, device=None):
    """One WIT sector with its candidate quartets split across the ranks of
    ``group`` (NCCL on CUDA tensors); every rank returns the summed fields
    [5][case][ny][nx] (a device tensor) and the combined statistics."""
    import torch
    import torch.distributed as dist

    from . import wit

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    m = int(np.asarray(inp.modes).reshape(-1, 2).shape[0])
    count = wit.candidates(sector, m)

    def compute(b, e):
        out = wit.wit_sector(inp, sector, device=device, as_numpy=False, q_range=(b, e))
        planes = torch.stack([out.fields[k] for k in wit.FIELDS])
        return planes, out.stats

    def reduce_sum(planes):
        if world > 1:
            dist.all_reduce(planes, op=dist.ReduceOp.SUM, group=group)
        return planes

    def gather(stats):
        if world == 1:
            return [stats]
        got = [None] * world
        dist.all_gather_object(got, stats, group=group)
        return got

    return wit_sharded(compute, reduce_sum, gather, count, rank, world)


def eta44_distributed(spectra, *, dk: float, depth: float, peak_depth: float, rank_gl: int,
                      group=None, device=None, output: str = "complex"):
    """eta44 of one or more spectra with the outer GL nodes split across the
    ranks of ``group`` (NCCL on CUDA tensors).  Every rank returns the fields."""
    import torch
    import torch.distributed as dist

    from . import _lib
    from .api import _engine_call, _status_error
    from .eta44 import Eta44Plan, _box

    spectra = np.asarray(spectra, dtype=np.complex128)
    if spectra.ndim == 2:
        spectra = spectra[None]
    units, n, _ = spectra.shape
    box = _box(np.abs(spectra).max(axis=0))
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    dev = torch.device(device if device is not None else "cuda")
    out_mode = _lib.OUT_REAL if output == "real" else _lib.OUT_COMPLEX
    desc = _lib.Eta44Desc(n=n, dk=dk, depth=depth, peak_depth=peak_depth, rank=rank_gl,
                          nodes=None, weights=None, box_x0=box[0], box_y0=box[1], box_w=box[2],
                          box_h=box[3], max_units=1, output=out_mode)
    plan = Eta44Plan(desc, dev)
    b4 = (4 * (box[3] - 1) + 1, 4 * (box[2] - 1) + 1)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    spec = torch.from_numpy(np.ascontiguousarray(spectra)).to(dev)
    status = torch.zeros(units, dtype=torch.int32, device=dev)

    def zeros():
        return torch.zeros((units,) + b4, dtype=torch.complex128, device=dev)

    def compute_partial(b, e):
        part = zeros()
        _engine_call(lib.gl_eta44_execute_partial(
            plan.handle, units, C.c_void_p(spec.data_ptr()), _lib.SPECTRA_FULL, b, e,
            C.c_void_p(part.data_ptr()), C.c_void_p(plan._ws_ptr()), C.c_size_t(plan.workspace_bytes),
            C.c_void_p(status.data_ptr()), C.c_void_p(stream)))
        return part

    def reduce_sum(part):
        if world > 1:
            dist.all_reduce(torch.view_as_real(part), op=dist.ReduceOp.SUM, group=group)
        return part

    def finalize(total):
        dtype = torch.float64 if out_mode == _lib.OUT_REAL else torch.complex128
        out = torch.empty((units, n, n), dtype=dtype, device=dev)
        _engine_call(lib.gl_eta44_finalize(
            plan.handle, units, C.c_void_p(total.data_ptr()), C.c_void_p(out.data_ptr()),
            C.c_void_p(plan._ws_ptr()), C.c_size_t(plan.workspace_bytes), C.c_void_p(stream)))
        return out

    out = eta44_sharded(compute_partial, reduce_sum, finalize, zeros, rank, rank_gl, world)
    st = status.cpu().numpy()
    if np.any(st != 0):
        raise _status_error(int(st[st != 0][0]))
    return out.cpu().numpy()
