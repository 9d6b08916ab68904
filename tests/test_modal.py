"""Single-direction time path (the reference's modal GL resolvent,
``python/src/green_laplace/modal_time.py`` + ``_eta20.py``): the CPU oracle
against the reference's golden vectors, and the GPU engine against both."""

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import gl_modal as M

GOLD = dict(np.load(Path(__file__).resolve().parent / "golden" / "modal_time.npz"))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _kw(tag):
    kw = json.loads(str(GOLD[tag + "/kw"]))
    if isinstance(kw.get("modal_points"), list):
        kw["modal_points"] = tuple(kw["modal_points"])
    if "eta20_grid" in kw:
        kw["eta20_grid"] = tuple(kw["eta20_grid"])
    return kw


def _matlab_m3():
    g = GOLD
    return dict(depth=float(g["m3/depth"]), gravity=float(g["m3/gravity"]),
                omega_max=float(g["m3/omega_max"]), energy_fraction=1.0,
                quadrature_rank=int(g["m3/rank"]), order=3, modal_points=int(g["m3/modal_points"]),
                modal_limit=float(g["m3/modal_limit"]), include_eta20=False)


def _matlab_e20():
    g = GOLD
    period = len(g["e20/time"]) * (g["e20/time"][1] - g["e20/time"][0])
    return dict(depth=float(g["e20/depth"]), gravity=float(g["e20/gravity"]),
                omega_max=2 * np.pi * 8 / period + 1e-12, energy_fraction=1.0, order=2,
                modal_points=512, include_eta20=True, eta20_rank=int(g["e20/rank"]),
                eta20_grid=tuple(int(x) for x in g["e20/grid"]))


def test_oracle_matches_matlab_fixtures():
    """The reference's own bars: 3e-13 (modal order 3), 8e-11 (eta20)
    (python/tests/test_temporal.py:25-26, 54)."""
    _, c, _ = M.modal_timeseries(GOLD["m3/eta1"], GOLD["m3/time"], **_matlab_m3())
    assert rel(c["eta22"], GOLD["m3/eta22"]) < 3e-13
    assert rel(c["eta33"], GOLD["m3/eta33"]) < 3e-13
    _, c, _ = M.modal_timeseries(GOLD["e20/eta1"], GOLD["e20/time"], **_matlab_e20())
    assert rel(c["eta20"], GOLD["e20/eta20"]) < 8e-11


@pytest.mark.parametrize("tag", ["ladder3", "broad3", "o2e20"])
def test_oracle_matches_reference_python(tag):
    eta, c, audit = M.modal_timeseries(GOLD[tag + "/eta1"], GOLD[tag + "/time"], **_kw(tag))
    assert audit["levels"] == list(GOLD[tag + "/levels"])
    for k in ("eta11", "eta22", "eta33", "eta20"):
        if f"{tag}/{k}" in GOLD:
            assert rel(c[k], GOLD[f"{tag}/{k}"]) < 1e-14, k
    assert rel(eta, GOLD[tag + "/eta"]) < 1e-14


# ---------------------------------------------------------------------------
# GPU: the engine's modal path (gl_modal_level, gl_eta20_level)
# ---------------------------------------------------------------------------


@pytest.mark.gpu
def test_engine_matches_matlab_fixtures():
    from gl_engine import modal

    r = modal.reconstruct_unidirectional_modal_timeseries(GOLD["m3/eta1"], GOLD["m3/time"],
                                                          **_matlab_m3())
    e22, e33 = rel(r.components["eta22"], GOLD["m3/eta22"]), rel(r.components["eta33"], GOLD["m3/eta33"])
    print(f"MATLAB modal order 3: eta22 {e22:.2e}, eta33 {e33:.2e}")
    assert e22 < 3e-13 and e33 < 3e-13
    r = modal.reconstruct_unidirectional_timeseries(GOLD["e20/eta1"], GOLD["e20/time"], **_matlab_e20())
    e20 = rel(r.components["eta20"], GOLD["e20/eta20"])
    print(f"MATLAB eta20: {e20:.2e}")
    assert e20 < 8e-11


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["ladder3", "broad3", "o2e20"])
def test_engine_matches_reference_python(tag):
    from gl_engine import modal

    r = modal.reconstruct_unidirectional_modal_timeseries(GOLD[tag + "/eta1"], GOLD[tag + "/time"],
                                                          **_kw(tag))
    assert [lv["modal_points"] for lv in r.audit["levels"]] == list(GOLD[tag + "/levels"])
    for k in ("eta11", "eta22", "eta33", "eta20"):
        if f"{tag}/{k}" in GOLD:
            err = rel(r.components[k], GOLD[f"{tag}/{k}"])
            print(f"{tag} {k}: {err:.2e}")
            assert err < 1e-12, k
    assert not r.audit["auxiliary_space_domain"]


@pytest.mark.gpu
def test_engine_four_step_axis_matches_oracle():
    """q-axes above 4096 nodes take the two-pass (four-step) transform; the
    level must equal the oracle's single-transform result."""
    from gl_engine import modal

    kw = dict(depth=1.0, omega_max=2 * np.pi * 24 / (512 * 0.2) + 1e-12, energy_fraction=1.0,
              quadrature_rank=4, order=3, modal_points=8192, include_eta20=False)
    eta1, t = GOLD["ladder3/eta1"], GOLD["ladder3/time"]
    _, c, _ = M.modal_timeseries(eta1, t, **kw)
    r = modal.reconstruct_unidirectional_modal_timeseries(eta1, t, **kw)
    for k in ("eta22", "eta33"):
        err = rel(r.components[k], c[k])
        print(f"four-step P=8192 {k}: {err:.2e}")
        assert err < 1e-12, k
