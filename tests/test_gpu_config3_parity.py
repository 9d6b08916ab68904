"""The uneven batch (64 sea states of the seeded batch workload: grids
128^2..1024^2, orders 2-3, ranks 2-8, depths 10-100 m) checked against the
oracle, one sea state per (grid, order, rank) class, through the batch
runner's captured CUDA graph -- the same path the batch benchmark times.

Every class is checked at 128^2, 256^2 and 512^2.  At 1024^2 the order-2
classes and order-3 GL4/GL4 are checked; order 3 at (6, 6) and (8, 8) on
1024^2 would take the single-threaded oracle minutes per snapshot, and those
rank pairs are covered by the 512^2 classes and by the reference's own
fields in test_gpu_rank_pairs.py.  Bounds: per case, from the oracle's
roundoff spread (parity_bounds).  The oracle's base and perturbed runs go to
a spawned process pool, one task each.
"""

import multiprocessing as mp

import numpy as np
import pytest
import torch

from gl_engine import batch
from parity_bounds import PERTURBATIONS, check_fields, oracle_surface_with_spread, rel

pytestmark = pytest.mark.gpu


def _classes():
    items = batch.config3_items()
    picked = {}
    for it in items:
        key = (it.nx, it.coeffs.order, int(it.coeffs.options["eta22_rank"]))
        if key in picked:
            continue
        if it.nx == 1024 and it.coeffs.order == 3 and it.inner_rank > 4:
            continue
        picked[key] = it
    return picked


def test_config3_classes_match_oracle_through_the_graph():
    picked = _classes()
    assert len(picked) >= 24
    items = []
    for key, it in sorted(picked.items()):
        # one snapshot per class (the oracle's cost), still through the graph
        items.append(batch.BatchItem(**{**it.__dict__, "times": np.asarray(it.times[:1])}))
    jobs = []
    for it in items:
        c = it.coeffs
        jobs.append(dict(order=c.order, gravity=c.g, depth=c.h, a=c.a, b=c.b, kx=c.kx, ky=c.ky,
                         eta22_rank=int(c.options["eta22_rank"]), inner=it.inner_rank,
                         outer=it.outer_rank, lx=it.lx, ly=it.ly, n=it.nx, t=float(it.times[0]),
                         names=tuple(it.components)))
    kinds = ("base",) + PERTURBATIONS
    tasks = [dict(job, perturbation=k) for job in jobs for k in kinds]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(32, mp.cpu_count())) as pool:
        pending = pool.map_async(oracle_surface_with_spread, tasks, chunksize=1)
        runner = batch.BatchRunner(items, output="complex")
        runner.capture()
        runner.replay()
        torch.cuda.synchronize()
        runner.check()
        runs = pending.get()
    results = []
    for c in range(len(jobs)):
        base, alts = runs[c * len(kinds)], runs[c * len(kinds) + 1:(c + 1) * len(kinds)]
        results.append((base, {k: max(rel(a[k], base[k]) for a in alts) for k in base}))
    for (it, names, out), (ref, spread) in zip(runner.outputs(), results):
        got = out[0].cpu().numpy()
        engine = {nm: got[k] for k, nm in enumerate(names)}
        label = f"{it.nx}^2 order {it.coeffs.order} rank {it.coeffs.options['eta22_rank']}" \
                f" GL{it.inner_rank}/{it.outer_rank}"
        check_fields(engine, ref, spread, label)
