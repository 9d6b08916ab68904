"""Even reference grids that are not powers of two.

The reference takes any even Nx, Ny (``python/src/green_laplace/_spectral.py:
9-16``; ``src/gl_spectral_surface.m:115-121``).  The engine runs sizes whose
prime factors are 2, 3 and 5: its product stages stay on compact power-of-two
grids covering their boxes, and the final transforms run at Nx x Ny through
the generic-length kernels.  Orders 2 and 3 against the oracle at square and
rectangular sizes, per-case bounds from the oracle's roundoff spread.
"""

import numpy as np
import pytest

import gl_engine
from parity_bounds import check_fields, oracle_fields_with_spread

pytestmark = pytest.mark.gpu


def _state(nx, ny, order, seed):
    """24 modes on the lattice of an (2 nx) m x (2 ny) m domain, h = 20 m,
    mode numbers mx in [3, 9], |my| <= 4 (alias-safe at order 3 on every grid
    below, kh > 0.5)."""
    rng = np.random.default_rng(seed)
    lx, ly = 2.0 * nx, 2.0 * ny
    cells = set()
    while len(cells) < 24:
        cells.add((int(rng.integers(3, 10)), int(rng.integers(-4, 5))))
    m = np.array(sorted(cells), dtype=float)
    kx, ky = m[:, 0] * 2 * np.pi / lx, m[:, 1] * 2 * np.pi / ly
    amp = 0.05 / np.sqrt(len(m))
    a, b = amp * rng.standard_normal(len(m)), amp * rng.standard_normal(len(m))
    return dict(gravity=9.81, depth=20.0, a=a, b=b, kx=kx, ky=ky, lx=lx, ly=ly)


@pytest.mark.parametrize("nx,ny,order", [(96, 96, 2), (96, 96, 3), (160, 160, 3), (192, 192, 2),
                                         (384, 384, 3), (96, 128, 3), (240, 80, 2)])
def test_non_power_of_two_grids_match_oracle(nx, ny, order):
    st = _state(nx, ny, order, seed=nx + ny + order)
    t = 0.6
    args = (st["gravity"], st["depth"], st["a"], st["b"], st["kx"], st["ky"])
    c = gl_engine.gl_spectral_coefficients(order, *args, 0, 0, {"eta22_rank": 4})
    _, _, _, _, comps, _ = gl_engine.gl_spectral_surface(c, st["lx"], st["ly"], nx, ny, t)
    ref, spread = oracle_fields_with_spread(order, *args, st["lx"], st["ly"], nx, ny, t,
                                            eta22_rank=4)
    plus = {k: v for k, v in ref.items() if k.endswith("_plus")}
    for k, v in plus.items():
        assert comps[k].shape == (ny, nx) == v.shape
    check_fields(comps, plus, spread, f"{nx}x{ny} order {order}")
