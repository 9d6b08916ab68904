"""The C-ABI library: builds, loads, exports every declared symbol, and its
host-only entry points (no GPU needed)."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from gl_engine import _lib
from gl_engine import api
from oracle import gl_oracle as O

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gl_engine.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(_lib.SIGNATURES), "binding misses a declared entry point"


def test_version_string():
    assert b"sm_100a" in _lib.load().gl_version()


@pytest.mark.parametrize("rank", list(range(1, 17)))
def test_native_gauss_laguerre_matches_oracle(rank):
    nodes, weights = api.gauss_laguerre_rule(rank)
    ref_nodes, ref_weights = O.gauss_laguerre(rank)
    assert np.allclose(nodes, ref_nodes, rtol=1e-13, atol=0)
    assert np.allclose(weights, ref_weights, rtol=1e-11, atol=1e-300)


def test_native_gauss_laguerre_rejects_bad_rank():
    with pytest.raises(ArithmeticError):
        api.gauss_laguerre_rule(0)


def test_native_dispersion_matches_oracle():
    omega = np.linspace(0.05, 3.0, 257)
    for depth in (1.0, 20.0, 100.0):
        q = api.dimensionless_wavenumber_from_frequency(omega, depth=depth, gravity=9.81)
        ref = O.dispersion_q(omega, depth, 9.81)
        assert np.allclose(q, ref, rtol=1e-14, atol=0)
        assert np.allclose(q * np.tanh(q), omega**2 * depth / 9.81, rtol=2e-13)


def test_native_dispersion_rejects_negative():
    with pytest.raises(ValueError):
        api.dimensionless_wavenumber_from_frequency([-1.0], depth=1.0)


def _desc(**kw):
    d = dict(nx=64, ny=64, lx=2 * np.pi, ly=2 * np.pi, depth=1.0, gravity=9.81, order=3,
             components=0, eta22_rank=6, inner_rank=4, outer_rank=4,
             allow_below_model_parent_domain=0, box_x0=2, box_y0=0, box_w=2, box_h=2, grid=0,
             max_units=1, output=0)
    d.update(kw)
    return _lib.PlanDesc(**d)


@pytest.mark.parametrize("kw,status,text", [
    (dict(order=4), 1, "order"),
    (dict(nx=56), 2, "no prime factor above 5"),
    (dict(nx=63), 1, "even"),
    (dict(box_x0=0), 7, "strict-forward"),
    (dict(box_x0=12, box_w=1), 14, "cubic"),
    (dict(order=2, box_x0=16, box_w=1, eta22_rank=6), 14, "quadratic"),
    (dict(box_x0=40, box_w=1), 13, "Nyquist"),
    (dict(inner_rank=5), 16, "rank"),
    (dict(order=2, eta22_rank=17), 16, "eta22_rank"),
    (dict(depth=-1.0), 1, "depth"),
    (dict(max_units=0), 1, "max_units"),
])
def test_plan_validation_errors_before_any_device_work(kw, status, text):
    lib = _lib.load()
    handle = C.c_void_p()
    st = lib.gl_plan_create(C.byref(handle), C.byref(_desc(**kw)))
    assert st == status
    assert text in _lib.last_error()
    assert not handle.value


def test_null_arguments_are_rejected():
    lib = _lib.load()
    assert lib.gl_plan_create(None, None) == 1
    assert lib.gl_execute(None, 1, None, 0, None, None, 0, None, None) == 1
    assert lib.gl_workspace_size(None, None) == 1
    assert lib.gl_plan_set_lanes(None, 2) == 1
    assert lib.gl_plan_set_tuning(None, None) == 1


@pytest.mark.parametrize("nx,ny", [(112, 112), (64, 98), (4100, 64), (8, 8)])
def test_plan_rejects_grids_outside_the_supported_sizes(nx, ny):
    """Sizes with a prime factor above 5, beyond 4096 or below 16 are refused
    before any device work (so this runs without a GPU)."""
    lib = _lib.load()
    desc = _lib.PlanDesc(nx=nx, ny=ny, lx=100.0, ly=100.0, depth=10.0, gravity=9.81, order=2,
                         components=0, eta22_rank=4, inner_rank=4, outer_rank=4,
                         allow_below_model_parent_domain=0, box_x0=1, box_y0=0, box_w=2, box_h=1,
                         grid=0, max_units=1, output=0)
    h = C.c_void_p()
    assert lib.gl_plan_create(C.byref(h), C.byref(desc)) == 2  # GL_ERR_UNSUPPORTED
    assert "no prime factor above 5" in _lib.last_error()
