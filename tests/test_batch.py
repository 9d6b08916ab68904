"""Uneven batches captured as one CUDA graph: replay equals eager execution
and the per-sea-state API, bit for bit."""

import numpy as np
import pytest
import torch

import gl_engine
from gl_engine import _lib, api, batch, seastate

pytestmark = pytest.mark.gpu


def _items():
    items = []
    rng = np.random.default_rng(5)
    for k, (n, order, rank) in enumerate([(64, 2, 2), (128, 3, 4), (64, 3, 6), (128, 2, 8)]):
        st = seastate.jonswap_sea_state(n=n, length=2.0 * n, depth=float(rng.uniform(10, 60)),
                                        hs=2.0, tp=8.0, modes=30, seed=k, order=order)
        c = gl_engine.gl_spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx,
                                               st.ky, 0, 0, {"eta22_rank": rank})
        r3 = rank if rank in (4, 6, 8) else 4
        comps = ("eta22", "psi22") if order == 2 else ("eta33", "psi33")
        items.append(batch.BatchItem(coeffs=c, lx=st.lx, ly=st.ly, nx=n, ny=n,
                                     times=rng.uniform(0, 60, 3), components=comps,
                                     inner_rank=r3, outer_rank=r3))
    return items


def test_graph_replay_equals_eager_and_single_calls():
    items = _items()
    runner = batch.BatchRunner(items)
    runner.run_eager()
    torch.cuda.synchronize()
    runner.check()
    eager = [t.clone() for _, _, t in runner.outputs()]
    runner.capture()
    for t in runner.outputs():
        t[2].zero_()
    runner.replay()
    torch.cuda.synchronize()
    runner.check()
    for (it, names, got), want in zip(runner.outputs(), eager):
        assert torch.equal(got, want)
        one = api.surface_batch_device(it.coeffs, it.lx, it.ly, it.nx, it.ny, it.times,
                                       components=list(it.components), output="real",
                                       max_units=len(it.times),
                                       order3_ranks=(it.inner_rank, it.outer_rank))
        assert one.names == names
        assert torch.equal(one.fields, got)


def test_concurrent_lanes_equal_one_lane():
    """States dealt to three concurrent lanes (own workspaces, parallel graph
    branches) give the one-lane results bit for bit."""
    items = _items()
    one = batch.BatchRunner(items, lanes=1)
    one.run_eager()
    three = batch.BatchRunner(items, lanes=3)
    assert three.lanes == 3 and len(set(three.lane_of)) == 3
    three.capture()
    for t in three.outputs():
        t[2].zero_()
    three.replay()
    torch.cuda.synchronize()
    one.check()
    three.check()
    for (_, _, a), (_, _, b) in zip(one.outputs(), three.outputs()):
        assert torch.equal(a, b)


def test_launch_shapes_do_not_change_results():
    """Every tuning of the row groups and column blocks gives the built-in
    launch's fields bit for bit (only the spreading over blocks changes)."""
    items = _items()
    ref = batch.BatchRunner(items, lanes=1)
    ref.run_eager()
    torch.cuda.synchronize()
    want = [t.clone() for _, _, t in ref.outputs()]
    for cfg in [(4, 8, 8), (16, 16, 4), (2, 12, 1), (8, 6, 16)]:
        for s in ref.staged:
            s.plan.set_tuning(*cfg)
        ref.run_eager()
        torch.cuda.synchronize()
        for (_, _, got), w in zip(ref.outputs(), want):
            assert torch.equal(got, w), cfg
    for s in ref.staged:
        s.plan.set_tuning(0, 0, 0)
    with pytest.raises(_lib.EngineError):
        ref.staged[0].plan.set_tuning(3, 0, 0)


def test_autotuner_picks_a_candidate():
    item = _items()[1]
    g = batch.autotune_group(item, candidates=(1, 3))
    assert g in (1, 3)
    assert batch.autotune_group(item, candidates=(1, 3)) == g  # cached
    tiles = batch.autotune_tiles(item)
    assert all(v in batch.TILE_CANDIDATES[n] for v, n in
               zip(tiles, ("pair_row_groups", "triple_row_groups", "col_block_columns")))
    k = batch.autotune_lanes(_items(), candidates=(1, 2))
    assert k in (1, 2)
    assert batch.autotune_lanes(_items(), candidates=(1, 2)) == k
