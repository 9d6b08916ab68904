"""Host-side logic of the drop-in API: the MATLAB validation identifiers,
the deposit bookkeeping and the sea-state generator (no GPU needed)."""

import numpy as np
import pytest

import gl_engine
from gl_engine import api, seastate
from oracle import gl_oracle as O

G = 9.81


def coeffs(order=3, **kw):
    base = dict(a=[.01, .006], b=[0, -.002], kx=[2, 3], ky=[0, 1])
    base.update(kw)
    return gl_engine.gl_spectral_coefficients(order, G, 1.0, base["a"], base["b"], base["kx"],
                                              base["ky"], 0.0, 0.0)


@pytest.mark.parametrize("args,ident", [
    (dict(kx=[0.5, 3]), "green_laplace:Order3Domain"),
    (dict(kx=[-2, 3]), "green_laplace:Support"),
    (dict(a=[0, 0], b=[0, 0]), "green_laplace:ZeroInput"),
    (dict(a=[np.nan, 1]), "green_laplace:Components"),
    (dict(a=[1, 2, 3]), "green_laplace:ComponentSize"),
])
def test_coefficient_identifiers(args, ident):
    with pytest.raises(gl_engine.GLError) as e:
        coeffs(**args)
    assert e.value.identifier == ident


def test_uniform_current_and_options():
    with pytest.raises(gl_engine.GLError) as e:
        gl_engine.gl_spectral_coefficients(2, G, 1.0, [1], [0], [2], [0], 0.1, 0.0)
    assert e.value.identifier == "green_laplace:UniformCurrent"
    with pytest.raises(gl_engine.GLError) as e:
        gl_engine.gl_spectral_coefficients(2, G, 1.0, [1], [0], [2], [0], 0, 0, {"bogus": 1})
    assert e.value.identifier == "green_laplace:UnknownOption"
    with pytest.raises(gl_engine.GLError) as e:
        gl_engine.gl_spectral_coefficients(2, G, 1.0, [1], [0], [2], [0], 0, 0, {"sector": "x"})
    assert e.value.identifier == "green_laplace:Sector"
    with pytest.raises(gl_engine.GLError) as e:
        gl_engine.gl_spectral_coefficients(2, G, 1.0, [1], [0], [0.2], [0], 0, 0)
    assert e.value.identifier == "green_laplace:Order2Domain"


def test_coefficients_fields_match_oracle():
    c = coeffs()
    o = O.spectral_coefficients(3, G, 1.0, [.01, .006], [0, -.002], [2, 3], [0, 1])
    assert c.api == "green-laplace-spectral-v1"
    assert np.array_equal(c.omega, o["omega"])
    assert c.peak_depth == o["peak_depth"]
    assert c.options["eta22_rank"] == 6


def test_deposit_bookkeeping_groups_coincident_modes():
    c = gl_engine.gl_spectral_coefficients(2, G, 1.0, [.01, .002, .003], [0, .001, 0],
                                           [2, 3, 2], [0, 1, 0], 0, 0)
    dep = api.prepare_deposit(c, 2 * np.pi, 2 * np.pi, 64, 64)
    assert dep.box == (2, 0, 2, 2)
    assert list(dep.seg_offsets) == [0, 2, 3]
    assert list(dep.seg_bins) == [0, 3]
    # coincident modes stay in input order inside their segment
    assert np.allclose(dep.ab[:4], [.01, 0, .003, 0])


def test_deposit_off_grid_and_nyquist():
    c = gl_engine.gl_spectral_coefficients(2, G, 1.0, [.01], [0], [2.3], [0], 0, 0)
    with pytest.raises(gl_engine.GLError) as e:
        api.prepare_deposit(c, 2 * np.pi, 2 * np.pi, 64, 64)
    assert e.value.identifier == "green_laplace:OffGridComponent"
    c = gl_engine.gl_spectral_coefficients(2, G, 1.0, [.01], [0], [32], [0], 0, 0)
    with pytest.raises(gl_engine.GLError) as e:
        api.prepare_deposit(c, 2 * np.pi, 2 * np.pi, 64, 64)
    assert e.value.identifier == "green_laplace:Nyquist"


def test_matlab_round_half_away_from_zero():
    assert list(api._matlab_round(np.array([0.5, 1.5, -0.5, -1.5, 2.4]))) == [1, 2, -1, -2, 2]


@pytest.mark.parametrize("maker,order", [(seastate.config1, 2), (seastate.config2, 3)])
def test_seastate_configs_are_admissible(maker, order):
    st = maker(0)
    dk = 2 * np.pi / st.lx
    mx = np.rint(st.kx / dk)
    my = np.rint(st.ky / dk)
    assert np.all(mx >= 1)
    assert np.max(order * np.abs(mx)) < st.nx / 2 and np.max(order * np.abs(my)) < st.ny / 2
    kh = np.hypot(st.kx, st.ky) * st.depth
    assert np.all(kh > 0.5) if order == 3 else np.all(kh >= 0.3)
    assert len(set(zip(mx, my))) == st.modes
    var = np.sum(st.a**2 + st.b**2) / 2
    assert 0.2 < var / ((2.0 if order == 2 else 3.0) ** 2 / 16) < 5
    # seeded determinism
    st2 = maker(0)
    assert np.array_equal(st.a, st2.a)
