"""Multi-rank orchestration on CPU (gloo, world size 2) and its single-GPU
equivalence: units shard without overlap, and outer-node sharding of eta44
with one all-reduce reproduces the monolithic field."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gl_engine import parallel
from oracle import gl_eta44 as OE
from oracle import gl_oracle as O


def test_split_range_partitions_exactly():
    for count in (0, 1, 5, 6, 10, 64):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                b, e = parallel.split_range(count, r, world)
                assert 0 <= b <= e <= count
                seen.extend(range(b, e))
            assert seen == list(range(count))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spectrum():
    rng = np.random.default_rng(3)
    n = 32
    s = np.zeros((n, n), dtype=complex)
    for mx, my in ((1, 0), (2, 1), (3, -1), (2, -2)):
        s[my % n, mx] = n * n * 0.02 * (rng.standard_normal() + 1j * rng.standard_normal())
    return s


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = _spectrum()
        nodes, weights = O.gauss_laguerre(3)
        state = {}

        def compute_partial(b, e):
            out, m4 = OE.eta44_partial(s, 0.25, 1.0, 1.0, nodes, weights, set(range(b, e)))
            state["m4"] = m4
            return torch.from_numpy(out)

        def zeros():
            state["m4"] = OE.Grid(s, 0.25, 1.0, 1.0, nodes, weights).m4
            return torch.zeros(s.shape, dtype=torch.complex128)

        def reduce_sum(part):
            dist.all_reduce(torch.view_as_real(part), op=dist.ReduceOp.SUM)
            return part

        def finalize(total):
            return OE.eta44_finalize(total.numpy(), state["m4"])

        field = parallel.eta44_sharded(compute_partial, reduce_sum, finalize, zeros, rank, 3, world)
        # unit sharding with max-over-ranks timing
        mine = parallel.shard_units(10, rank, world)
        t = torch.tensor([float(mine.stop - mine.start)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((field, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_eta44_outer_sharding_with_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    field, tmax = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nodes, weights = O.gauss_laguerre(3)
    full = OE.eta44(_spectrum(), 0.25, 1.0, 1.0, nodes, weights)
    assert np.linalg.norm(field - full) / np.linalg.norm(full) < 1e-13
    assert tmax == 5.0


@pytest.mark.gpu
def test_eta44_partials_sum_to_monolithic_on_one_gpu():
    """Sequential stand-in for the multi-GPU split: the partials of a
    partition of the outer nodes, summed and finalised, equal the one-shot field."""
    from gl_engine import eta44 as E44
    import ctypes as C
    from gl_engine import _lib
    from gl_engine.api import _engine_call

    s = _spectrum()
    rank = 4
    full = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank)
    box = E44._box(np.abs(s))
    desc = _lib.Eta44Desc(n=32, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank, nodes=None,
                          weights=None, box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3],
                          max_units=1, output=_lib.OUT_COMPLEX)
    plan = E44.Eta44Plan(desc, torch.device("cuda"))
    lib = _lib.load()
    dev = torch.device("cuda")
    spec = torch.from_numpy(s[None].copy()).to(dev)
    b4 = (4 * (box[3] - 1) + 1, 4 * (box[2] - 1) + 1)
    total = torch.zeros((1,) + b4, dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for b, e in ((0, 1), (1, 3), (3, 4)):
        part = torch.zeros_like(total)
        _engine_call(lib.gl_eta44_execute_partial(plan.handle, 1, C.c_void_p(spec.data_ptr()), 0, b,
                                                  e, C.c_void_p(part.data_ptr()),
                                                  C.c_void_p(plan._ws_ptr()),
                                                  C.c_size_t(plan.workspace_bytes), None,
                                                  C.c_void_p(stream)))
        total += part
    out = torch.empty((1, 32, 32), dtype=torch.complex128, device=dev)
    _engine_call(lib.gl_eta44_finalize(plan.handle, 1, C.c_void_p(total.data_ptr()),
                                       C.c_void_p(out.data_ptr()), C.c_void_p(plan._ws_ptr()),
                                       C.c_size_t(plan.workspace_bytes), C.c_void_p(stream)))
    got = out[0].cpu().numpy()
    assert np.linalg.norm(got - full) / np.linalg.norm(full) < 1e-13


def _toy_wit_range(b, e, ny=8, nx=8):
    """A stand-in share of a quartet sum for the host logic: candidate q adds
    a value of its own to one bin, and the statistics count and bound it."""
    out = torch.zeros((5, 1, ny, nx), dtype=torch.complex128)
    res, det = 0.0, float("inf")
    for q in range(b, e):
        out[q % 5, 0, (3 * q) % ny, (7 * q) % nx] += complex(np.sin(q), np.cos(0.5 * q))
        res = max(res, abs(np.sin(1.3 * q)))
        det = min(det, 1.0 + abs(np.cos(0.7 * q)))
    stats = {"candidates": e - b, "kept": (e - b) // 2, "near": (e - b) // 3,
             "strict_zero_output": 0, "strict_zero_intermediate": e - b - (e - b) // 2,
             "max_residual": res, "max_strict_zero_source": 0.0, "min_detuning": det}
    return out, stats


def _wit_worker(rank, world, port, q, count):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def reduce_sum(planes):
            dist.all_reduce(torch.view_as_real(planes), op=dist.ReduceOp.SUM)
            return planes

        def gather(stats):
            got = [None] * world
            dist.all_gather_object(got, stats)
            return got

        fields, stats = parallel.wit_sharded(_toy_wit_range, reduce_sum, gather, count, rank, world)
        q.put((rank, fields.numpy(), stats))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("count", [37, 1])
def test_wit_quartet_sharding_with_gloo_world2(count):
    """Two gloo ranks split the candidates, sum their planes with one
    all-reduce and combine their statistics: both equal the one-rank sum
    (count 1 leaves rank 1 an empty share)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_wit_worker, args=(r, 2, port, q, count)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one, one_stats = _toy_wit_range(0, count)
    expect = parallel.combine_wit_stats([one_stats])
    for _, fields, stats in got:
        assert np.allclose(fields, one.numpy(), rtol=0, atol=1e-12)
        assert stats == expect
