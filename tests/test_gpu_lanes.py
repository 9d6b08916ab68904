"""Concurrent lanes of one plan (gl_plan_set_lanes): the unit groups of a
gl_execute call spread over the plan's streams give the one-lane outputs bit
for bit, eagerly and replayed from a captured CUDA graph, for ragged unit
counts; bad lane counts are refused."""

import ctypes as C

import numpy as np
import pytest
import torch

import gl_engine
from gl_engine import _lib, api, seastate

pytestmark = pytest.mark.gpu


def _case(n=128, order=3, units=7, seed=3):
    st = seastate.jonswap_sea_state(n=n, length=2.0 * n, depth=25.0, hs=2.0, tp=8.0, modes=40,
                                    seed=seed, order=order)
    c = gl_engine.gl_spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    times = np.linspace(0.0, 30.0, units)
    dep = api.prepare_deposit(c, st.lx, st.ly, n, n)
    comps = _lib.COMP_ETA33 | _lib.COMP_PSI33 if order == 3 else _lib.COMP_ETA22 | _lib.COMP_PSI22
    desc = api.get_plan(nx=n, ny=n, lx=st.lx, ly=st.ly, depth=st.depth, gravity=st.gravity,
                        order=order, components=comps, eta22_rank=6, allow_below=False,
                        box=dep.box, grid=_lib.GRID_COMPACT, max_units=4, output=_lib.OUT_REAL,
                        device=torch.device("cuda")).desc
    dev = torch.device("cuda")
    d = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    w, h = dep.box[2], dep.box[3]
    spectra = torch.empty((units, h, w, 2), dtype=torch.float64, device=dev)
    plan = api.Plan(desc, dev)
    plan.deposit(units, d(dep.seg_offsets, torch.int32), d(dep.seg_bins, torch.int32),
                 d(dep.ab, torch.float64), d(dep.omega, torch.float64), d(times, torch.float64),
                 spectra, torch.cuda.current_stream().cuda_stream)
    return desc, spectra, n


def _run(plan, spectra, n, units):
    out = torch.full((units, 2, n, n), float("nan"), dtype=torch.float64, device="cuda")
    status = torch.full((units,), -1, dtype=torch.int32, device="cuda")
    plan.execute(units, spectra, _lib.SPECTRA_BOX, out, status,
                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out, status


@pytest.mark.parametrize("order", [2, 3])
def test_lanes_equal_one_lane_bitwise(order):
    desc, spectra, n = _case(order=order)
    units = spectra.shape[0]
    ref, st_ref = _run(api.Plan(desc, torch.device("cuda")), spectra, n, units)
    assert int(st_ref.abs().sum()) == 0
    assert torch.isfinite(ref).all()
    for lanes in (2, 3, 4, 8):
        plan = api.Plan(desc, torch.device("cuda"))
        ws_one = plan.workspace_bytes
        plan.set_lanes(lanes)
        # lanes regions of ceil(max_units / lanes) units: about one group's size
        assert plan.workspace_bytes <= 2 * ws_one
        for units_run in (units, 1, 5):
            got, st = _run(plan, spectra, n, units_run)
            assert int(st.abs().sum()) == 0
            assert torch.equal(got, ref[:units_run]), (lanes, units_run)


def test_lanes_inside_a_captured_graph():
    desc, spectra, n = _case()
    units = spectra.shape[0]
    ref, _ = _run(api.Plan(desc, torch.device("cuda")), spectra, n, units)
    plan = api.Plan(desc, torch.device("cuda"))
    plan.set_lanes(2)
    out = torch.zeros((units, 2, n, n), dtype=torch.float64, device="cuda")
    status = torch.zeros(units, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # eager once: kernel attributes, first-use set-up
        plan.execute(units, spectra, _lib.SPECTRA_BOX, out, status, side.cuda_stream)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        plan.execute(units, spectra, _lib.SPECTRA_BOX, out, status, side.cuda_stream)
    out.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert int(status.abs().sum()) == 0
    assert torch.equal(out, ref)
    del g


def test_lane_counts_outside_the_range_are_refused():
    desc, _, _ = _case(units=1)
    plan = api.Plan(desc, torch.device("cuda"))
    lib = _lib.load()  # GL_ERR_INVALID_ARGUMENT = 1
    for bad in (0, -1, _lib.MAX_LANES + 1):
        assert lib.gl_plan_set_lanes(plan.handle, bad) == 1
    assert "lanes must be" in _lib.last_error()
    assert lib.gl_plan_set_lanes(C.c_void_p(), 2) == 1
