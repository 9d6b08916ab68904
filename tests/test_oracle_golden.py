"""The CPU oracle against the reference's golden vectors (no GPU needed).

* MATLAB fixtures of the reference (python/tests/test_spatial.py:16-65),
  with the reference's own tolerances;
* outputs of the reference Python package on seeded inputs
  (tests/golden/make_golden.py), and of its order-3 graph at inner / outer
  GL rank pairs other than GL4/GL4 (tests/golden/make_rank_pairs.py).
"""

import math
from pathlib import Path

import numpy as np
import pytest

from oracle import gl_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def matlab():
    return dict(np.load(GOLD / "matlab_fixtures.npz"))


@pytest.fixture(scope="module")
def refpy():
    return dict(np.load(GOLD / "reference_python.npz"))


@pytest.fixture(scope="module")
def rank_pairs():
    return dict(np.load(GOLD / "order3_rank_pairs.npz"))


def _fixture_run(m, tag, order):
    rank = int(m[f"{tag}/rank"]) if f"{tag}/rank" in m else 6
    time = float(m[f"{tag}/time"]) if f"{tag}/time" in m else 0.0
    return O.reconstruct_directional_field(
        m[f"{tag}/eta1"], lx=float(m[f"{tag}/lx"]), ly=float(m[f"{tag}/ly"]),
        depth=float(m[f"{tag}/depth"]), gravity=float(m[f"{tag}/gravity"]), time=time,
        order=order, eta22_rank=rank)


def test_matlab_eta22_fixture(matlab):
    r = _fixture_run(matlab, "eta22", 2)
    assert rel(r["eta11"], matlab["eta22/eta1"]) < 2e-13
    assert rel(r["eta22"], matlab["eta22/eta22"]) < 2e-12
    assert rel(r["psi11"], matlab["eta22/psi11"]) < 2e-13
    assert rel(r["psi22"], matlab["eta22/psi22"]) < 3e-12


def test_matlab_order3_fixture(matlab):
    r = _fixture_run(matlab, "order3", 3)
    assert rel(r["eta33"], matlab["order3/eta33"]) < 5e-11
    assert rel(r["psi33"], matlab["order3/psi33"]) < 5e-11


def test_matlab_nonzero_time_fixture(matlab):
    r = _fixture_run(matlab, "time", 3)
    for c in ("eta11", "psi11", "eta22", "psi22", "eta33", "psi33"):
        assert rel(r[c], matlab[f"time/{c}"]) < 8e-11, c


@pytest.mark.parametrize("tag", ["fixture_t0", "fixture_t07", "jonswap64_o3", "jonswap64_o2",
                                 "jonswap128_o3"])
def test_oracle_matches_reference_python(refpy, tag):
    meta = refpy[f"{tag}/meta"]
    order, g, h, lx, ly, nx, ny, t, rank = meta
    a, b, kx, ky = refpy[f"{tag}/modes"]
    coeffs = O.spectral_coefficients(int(order), g, h, a, b, kx, ky,
                                     options={"eta22_rank": int(rank)})
    out = O.spectral_surface(coeffs, lx, ly, int(nx), int(ny), t)
    keys = [k.split("/")[1] for k in refpy if k.startswith(tag + "/")]
    checked = 0
    for c in keys:
        if c in ("meta", "modes"):
            continue
        assert rel(out[c], refpy[f"{tag}/{c}"]) < 1e-14, c
        checked += 1
    assert checked >= 2


def test_two_stage_deposit_reproduces_matlab_fixture(matlab):
    """The restated deposit (gl_spectral_surface.m:123-149) on the fixture
    mode list reproduces the MATLAB eta11/eta33 fields."""
    coeffs = O.spectral_coefficients(3, 9.81, 1.0, [.01, .006], [0, -.002], [2, 3], [0, 1],
                                     options={"eta22_rank": 6})
    out = O.spectral_surface(coeffs, 2 * np.pi, 2 * np.pi, 64, 64, 0.0)
    assert rel(out["eta11"], matlab["order3/eta1"]) < 1e-14
    assert rel(out["eta33"], matlab["order3/eta33"]) < 5e-11
    assert rel(out["psi33"], matlab["order3/psi33"]) < 5e-11


def test_gauss_laguerre_moments():
    """quadrature known-answer (python/tests/test_quadrature.py:8-15)."""
    nodes, weights = O.gauss_laguerre(8)
    assert np.all(nodes > 0) and np.all(weights > 0)
    for d in range(16):
        assert np.isclose(np.sum(weights * nodes**d), math.factorial(d), rtol=3e-11)


def test_roundoff_floor_semantics():
    s = np.array([[1.0 + 0j, 1e-14, 0.5], [1e-12, 0.0, 2.0]])
    sup = np.array([[True, True, False], [True, True, True]])
    out = O.zero_below_roundoff_floor(s, sup)
    floor = 16 * np.finfo(float).eps * max(1.0, np.log2(s.size)) * 2.0
    assert out[0, 1] == 0 and out[0, 2] == 0.5 and out[1, 0] == (1e-12 if 1e-12 >= floor else 0)
    assert out[1, 2] == 2.0


def test_minkowski_support_matches_direct_sum():
    rng = np.random.default_rng(0)
    n = 32
    sup = np.zeros((n, n), dtype=bool)
    for _ in range(12):
        sup[rng.integers(-4, 5) % n, rng.integers(1, 6)] = True
    s2 = O.minkowski_support(sup, 2)
    ys, xs = np.nonzero(sup)
    direct = np.zeros_like(sup)
    for y1, x1 in zip(ys, xs):
        for y2, x2 in zip(ys, xs):
            direct[(y1 + y2) % n, (x1 + x2) % n] = True
    assert np.array_equal(s2, direct)


@pytest.mark.parametrize("inner,outer", [(6, 3), (8, 6), (4, 10), (12, 4), (6, 6), (8, 8),
                                         (10, 10)])
def test_oracle_order3_rank_pairs_match_reference(rank_pairs, inner, outer):
    """_order3.py:18-26 takes the inner and outer ranks as arguments; the
    oracle's order3 reproduces it at unequal rank pairs."""
    g, h, lx, ly, nx, ny, t = rank_pairs["meta"]
    a, b, kx, ky = rank_pairs["modes"]
    nx, ny = int(nx), int(ny)
    oc = O.spectral_coefficients(3, g, h, a, b, kx, ky)
    s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], h, lx, ly, nx, ny, t)
    kxg, kyg = O.fft_wavenumber_grid(lx, ly, nx, ny)
    e33, p33, audit = O.order3(s, h * kxg, h * kyg, inner_rank=inner, outer_rank=outer)
    assert audit["inner_quadrature_rank"] == inner and audit["outer_quadrature_rank"] == outer
    assert rel(e33, rank_pairs[f"gl{inner}_{outer}/eta33"]) < 1e-14
    assert rel(p33, rank_pairs[f"gl{inner}_{outer}/psi33"]) < 1e-14
