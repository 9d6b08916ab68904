"""Failure paths of the device graph, exercised without faulting the GPU.

* Bounded waits: the row stages stage their bank rows with bulk asynchronous
  copies completed on an mbarrier and wait on it with a clock budget.  The
  plan's wait test hook (gl_plan_set_wait_test) makes every order-2/3 row
  launch expect more bytes than its copies deliver, with a ~1 ms budget: the
  wait runs out, every unit reports GL_ERR_TIMEOUT, and the same plan then
  runs normally again (the context is intact) and still matches the oracle.
* Non-finite input: a NaN in one unit's spectrum is reported as
  green_laplace:Components for that unit only; the other unit is unaffected.
* Non-finite output: finite spectra whose cubic products overflow are
  reported as GL_ERR_NONFINITE by the final transform's output check.

Nothing here makes a kernel trap, fault or wait without a bound.
"""

import numpy as np
import pytest
import torch

import gl_engine
from gl_engine import _lib, api, seastate
from parity_bounds import check_fields, oracle_fields_with_spread

pytestmark = pytest.mark.gpu
ST = {name: code for code, name in _lib.STATUS_NAMES.items()}


def _setup(order, n=64, seed=2, times=(0.0, 0.9)):
    st = seastate.small_order3(seed=seed, n=n, modes=12)
    c = gl_engine.gl_spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 4})
    dep = api.prepare_deposit(c, st.lx, st.ly, n, n)
    dev = torch.device("cuda", 0)
    # a plan of its own (not the cached one other tests share): the hook is per plan
    box = dep.box
    desc = api.PlanDesc(nx=n, ny=n, lx=st.lx, ly=st.ly, depth=c.h, gravity=c.g, order=order,
                        components=api._components_for(order, None), eta22_rank=4, inner_rank=4,
                        outer_rank=4, allow_below_model_parent_domain=0, box_x0=box[0],
                        box_y0=box[1], box_w=box[2], box_h=box[3], grid=api.GRID_COMPACT,
                        max_units=len(times), output=api.OUT_COMPLEX)
    plan = api.Plan(desc, dev)
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
    spec = torch.empty((len(times), dep.box[3], dep.box[2], 2), dtype=torch.float64, device=dev)
    plan.deposit(len(times), t(dep.seg_offsets, torch.int32), t(dep.seg_bins, torch.int32),
                 t(dep.ab, torch.float64), t(dep.omega, torch.float64),
                 t(np.asarray(times, dtype=float), torch.float64), spec,
                 torch.cuda.current_stream(dev).cuda_stream)
    return st, c, plan, spec


def _run(plan, spec):
    dev = spec.device
    u = spec.shape[0]
    out = torch.empty((u, plan.info.n_components, plan.desc.ny, plan.desc.nx),
                      dtype=torch.complex128, device=dev)
    status = torch.zeros(u, dtype=torch.int32, device=dev)
    plan.execute(u, spec, api.SPECTRA_BOX, out, status, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), status.cpu().numpy()


@pytest.mark.parametrize("order", [2, 3])
def test_row_wait_runs_out_and_the_plan_recovers(order):
    st, c, plan, spec = _setup(order)
    lib = _lib.load()
    good, s0 = _run(plan, spec)
    assert np.all(s0 == 0)
    # ~1 ms of SM clocks per wait, 16 bytes that never arrive
    _lib.check(lib.gl_plan_set_wait_test(plan.handle, 16, 2_000_000))
    try:
        _, s1 = _run(plan, spec)
    finally:
        _lib.check(lib.gl_plan_set_wait_test(plan.handle, 0, 0))
    assert np.all(s1 == ST["GL_ERR_TIMEOUT"]), s1
    again, s2 = _run(plan, spec)
    assert np.all(s2 == 0)
    assert np.array_equal(again, good)
    # and the recovered result is still the oracle's
    ref, spread = oracle_fields_with_spread(order, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                            st.lx, st.ly, st.nx, st.ny, 0.0, eta22_rank=4)
    names = [_lib.COMP_NAMES[i] + "_plus" for i in plan.component_ids]
    check_fields({nm: again[0, k] for k, nm in enumerate(names)}, {nm: ref[nm] for nm in names},
                 spread, f"recovered order {order}")


def test_wait_hook_rejects_an_unbounded_request():
    _, _, plan, _ = _setup(2)
    lib = _lib.load()
    assert lib.gl_plan_set_wait_test(plan.handle, 16, 0) == ST["GL_ERR_INVALID_ARGUMENT"]
    assert lib.gl_plan_set_wait_test(None, 0, 0) == ST["GL_ERR_INVALID_ARGUMENT"]


def test_nan_input_is_reported_for_its_unit_only():
    _, _, plan, spec = _setup(3)
    good, _ = _run(plan, spec)
    bad = spec.clone()
    bad[1, bad.shape[1] // 2, 0, 0] = float("nan")
    out, status = _run(plan, bad)
    assert status[0] == 0
    assert status[1] == ST["GL_ERR_COMPONENTS"]
    assert np.array_equal(out[0], good[0])


def test_overflowing_products_are_reported_nonfinite():
    _, _, plan, spec = _setup(3)
    big = spec * 1e200  # finite input; its cubic products overflow
    assert torch.isfinite(big).all()
    _, status = _run(plan, big)
    assert np.all(status == ST["GL_ERR_NONFINITE"]), status
