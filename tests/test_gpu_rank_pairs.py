"""Order-3 GPU parity at the inner/outer GL rank pairs the graph runs.

``green_laplace_order3`` (``python/src/green_laplace/_order3.py:18-26``)
accepts inner ranks {4, 6, 8, 10, 12} and outer ranks {3, 4, 6, 8, 10}; its
unified API fixes GL4/GL4, and the uneven batch workload runs (6, 6) and
(8, 8).  The golden fields are the reference's own outputs at each pair
(``tests/golden/make_rank_pairs.py``).  The engine must match them within the
per-case bound of ``parity_bounds`` (4x the oracle's roundoff spread on the
same case, never looser than needed below the 1e-12 FP64 bar).
"""

from pathlib import Path

import numpy as np
import pytest

import gl_engine
from gl_engine import api
from parity_bounds import check_fields, oracle_surface_with_spread

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
PAIRS = [(4, 4), (6, 3), (8, 6), (4, 10), (12, 4), (6, 6), (8, 8), (10, 10)]


@pytest.fixture(scope="module")
def rank_pairs():
    return dict(np.load(GOLD / "order3_rank_pairs.npz"))


@pytest.mark.parametrize("inner,outer", PAIRS)
def test_engine_matches_reference_at_rank_pair(rank_pairs, inner, outer):
    g, h, lx, ly, nx, ny, t = rank_pairs["meta"]
    a, b, kx, ky = rank_pairs["modes"]
    n = int(nx)
    c = gl_engine.gl_spectral_coefficients(3, g, h, a, b, kx, ky)
    res = api.surface_batch_device(c, lx, ly, n, n, [t], components=["eta33", "psi33"],
                                   order3_ranks=(inner, outer))
    got = res.fields[0].cpu().numpy()
    engine = {"eta33": got[0], "psi33": got[1]}
    oracle, spread = oracle_surface_with_spread(dict(
        order=3, gravity=g, depth=h, a=a, b=b, kx=kx, ky=ky, eta22_rank=6, inner=inner,
        outer=outer, lx=lx, ly=ly, n=n, t=t, names=("eta33", "psi33")))
    key = f"gl{inner}_{outer}"
    if f"{key}/eta33" in rank_pairs:  # the reference's own fields
        ps = h * np.sqrt(g * h)
        ref = {"eta33": h * rank_pairs[f"{key}/eta33"], "psi33": ps * rank_pairs[f"{key}/psi33"]}
        for k in ref:  # the oracle is the reference here, bit for bit or nearly
            assert np.linalg.norm(oracle[k] - ref[k]) <= 1e-14 * np.linalg.norm(ref[k])
    else:
        ref = oracle
    check_fields(engine, ref, spread, f"GL{inner}/GL{outer}")
